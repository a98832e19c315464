// MATLAB-facing I/O of a multislice run (matio.cpp): input struct from a MAT-file, output struct
// to a MAT-file.
#pragma once

#include <memory>
#include <string>
#include <vector>

#include "matfile.hpp"
#include "multem_b200.h"

namespace mtb {
namespace matio {

// An input read from a MAT-file: the C ABI structs and the arrays they point to.
struct Input {
    mt_system_conf conf{};
    mt_input_multislice in{};
    std::vector<std::vector<double>> store;
};

// The struct variable `var` (the first struct variable when empty) of the MAT-file at `path`.
std::unique_ptr<Input> read_input(const std::string& path, const std::string& var);
// Writes the output struct of a run with output sizes d as variable `var` ("output_multislice"
// when empty).
void write_output(const std::string& path, const std::string& var, const mt_output_dims& d,
                  const mt_output_multislice& out, bool compress);

}  // namespace matio
}  // namespace mtb
