// MAT-file (level 5: MATLAB -v6 and -v7) reader and writer for the engine's MATLAB-facing entry
// points: the input struct that `multem_input.parameters.toStruct` produces and the output struct
// that ilc_multem returns (set_struct_multislice, mex_files_multem/ilc_multem.cu:382-481).
//
// Format (MathWorks, "MAT-File Format", level 5): a 128-byte header (text, subsystem offset,
// version 0x0100, endian indicator "IM" for little endian), then data elements, each an 8-byte tag
// (type, byte count) and its data padded to 8 bytes, or a "small" element (byte count <= 4 packed
// with the type into the first 4 bytes of the tag, data in the other 4). A variable is an
// miMATRIX element (array flags, dimensions, name, then the data: real and imaginary parts of a
// numeric or char array, the field names and every element's fields of a struct array, the
// elements of a cell array); -v7 files wrap each variable in an miCOMPRESSED element (zlib).
// Numeric data may be stored in a narrower type than its class (MATLAB writes [1 2 3] as
// miUINT8); the reader converts every numeric, char and logical array to double.
// Not supported: big-endian files, sparse arrays, objects (classdef values: save the struct from
// toStruct instead), -v7.3 (HDF5) files, and variables over 2^31 bytes.
#pragma once

#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace mtb {
namespace mat {

enum Class : int {
    kCell = 1, kStruct = 2, kObject = 3, kChar = 4, kSparse = 5, kDouble = 6, kSingle = 7,
    kInt8 = 8, kUInt8 = 9, kInt16 = 10, kUInt16 = 11, kInt32 = 12, kUInt32 = 13, kInt64 = 14, kUInt64 = 15
};

struct Value {
    int cls = kDouble;
    bool complex = false;
    bool logical = false;
    std::vector<int64_t> dims{0, 0};       // MATLAB dimensions (at least two)
    std::vector<double> re, im;             // numeric, char (code points) and logical data, column-major
    std::vector<std::string> fields;        // struct: field names
    std::vector<Value> elems;               // struct: element e, field f at e * fields.size() + f; cell: elements

    size_t numel() const;
    bool is_struct() const { return cls == kStruct; }
    bool is_numeric() const { return cls != kStruct && cls != kCell && cls != kObject && cls != kSparse; }
    // field `name` of struct element e (nullptr when absent)
    const Value* field(const std::string& name, size_t e = 0) const;
    std::string str() const;                // char array as text

    static Value scalar(double v);
    static Value row(const std::vector<double>& v);                       // 1 x n
    static Value matrix(int64_t rows, int64_t cols, const double* re, const double* im = nullptr,
                        size_t im_stride = 1);                            // column-major data
    static Value string(const std::string& s);
    static Value struct_array(int64_t rows, int64_t cols, std::vector<std::string> fields);
    Value& at(size_t e, const std::string& name);                         // struct element field
};

using Variables = std::vector<std::pair<std::string, Value>>;

// Every variable of a level-5 MAT-file (throws mtb::Error MT_ERR_INVALID_ARG with a message on
// anything unreadable).
Variables read_file(const std::string& path);
// Writes a level-5 MAT-file; `compress` wraps each variable in a zlib-compressed element (-v7).
void write_file(const std::string& path, const Variables& vars, bool compress);

}  // namespace mat
}  // namespace mtb
