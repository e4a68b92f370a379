"""Records the mangled names of the reference's public C++ entry points
(its include/TensorBLAS.h:139-167: tc_syrk, tc_cumpsgemm_*, tc_ozimmu_*,
tc_trsm, tc_syr2k, tc_trmm, tc_symm) and of its extern "C" wrappers, read
with `nm` from the reference built from its own sources by oracle/Makefile:
oracle/_ref/libTensorBLAS_ref.so (plain and FP64 routines) and the
compile-only objects oracle/_ref/cxx_sym/tc_cumpsgemm_*.o (libcumpsgemm is
not vendored, so those are never linked; their handle type comes from the
declaration-only stub oracle/ref_stub/cumpsgemm/cumpsgemm.hpp).

    make -C oracle && python tests/golden/make_ref_symbols.py

writes tests/golden/ref_cxx_symbols.txt, which tests/test_abi.py compares
with the library's exported symbols.
"""
import glob
import os
import re
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
OUT = os.path.join(ROOT, "tests", "golden", "ref_cxx_symbols.txt")
PUBLIC = re.compile(r"^_Z\d+tc_(syrk|trsm|syr2k|trmm|symm|cumpsgemm_(syrk|trsm|syr2k|trmm|symm)|"
                    r"ozimmu_(syrk|trsm|syr2k|trmm))[A-Z]")
C_ABI = {"tc_syrk_wrapper", "tc_trsm_wrapper", "print_env"}


def reference_symbols(root=ROOT):
    ref = os.path.join(root, "oracle", "_ref")
    files = [os.path.join(ref, "libTensorBLAS_ref.so")] + sorted(glob.glob(os.path.join(ref, "cxx_sym", "*.o")))
    names = set()
    for f in files:
        if not os.path.exists(f):
            raise FileNotFoundError(f"{f}: build the reference first (make -C oracle)")
        args = ["nm", "-D", "--defined-only", f] if f.endswith(".so") else ["nm", "--defined-only", f]
        for line in subprocess.run(args, capture_output=True, text=True, check=True).stdout.splitlines():
            parts = line.split()
            if len(parts) == 3 and parts[1] == "T" and (PUBLIC.match(parts[2]) or parts[2] in C_ABI):
                names.add(parts[2])
    return sorted(names)


def main():
    names = reference_symbols()
    with open(OUT, "w") as f:
        f.write("\n".join(names) + "\n")
    print(f"{len(names)} symbols -> {OUT}")


if __name__ == "__main__":
    sys.exit(main())
