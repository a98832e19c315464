"""Lobato (0-12) coefficients, the Doyle-Turner / Peng / Kirkland coefficients (FEG_CL[t - 1], FEG_CNL[t - 1]
for potential_type t = 1..4), Peng's ionic coefficients (PENG_ION[(Z, charge index)]), mass numbers and atomic radii for Z = 1..103, read from the data file
the engine compiles in (multem_b200/csrc/atomic_params.inc, extracted from the reference's
src/atomic_data.hpp by multem_b200/csrc/gen_atomic_params.py). Test infrastructure only."""
import re
from pathlib import Path

_INC = Path(__file__).resolve().parents[1] / "multem_b200" / "csrc" / "atomic_params.inc"


def _parse():
    s = _INC.read_text()

    def table(name):
        body = re.search(name + r"\[103\]\[5\] = \{(.*?)\n\};", s, re.S).group(1)
        rows = re.findall(r"\{([^}]*)\}", body)
        return [[float(v) for v in r.split(",")] for r in rows]

    def vec(name, cast):
        body = re.search(name + r"\[103\] = \{([^}]*)\}", s).group(1)
        return [cast(v) for v in body.split(",")]

    def feg(name):
        body = re.search(name + r"\[4\]\[103\]\[6\] = \{(.*?)\n\};", s, re.S).group(1)
        rows = [[float(v) for v in r.split(",")] for r in re.findall(r"\{([^{}]*)\}", body)]
        return [rows[103 * t:103 * (t + 1)] for t in range(4)]

    def ions():
        body = re.search(r"kPengIon\[\d+\] = \{(.*?)\n\};", s, re.S).group(1)
        out = {}
        for m in re.finditer(r"\{(\d+), (\d+), \{([^}]*)\}, \{([^}]*)\}\}", body):
            out[(int(m.group(1)), int(m.group(2)))] = ([float(v) for v in m.group(3).split(",")],
                                                       [float(v) for v in m.group(4).split(",")])
        return out

    return (table("kLobatoCl"), table("kLobatoCnl"), vec("kMassNumber", int), vec("kAtomicRadius", float),
            feg("kFegCl"), feg("kFegCnl"), ions())


LOBATO_CL, LOBATO_CNL, MASS_NUMBER, ATOMIC_RADIUS, FEG_CL, FEG_CNL, PENG_ION = _parse()
