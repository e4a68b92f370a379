"""Records the reference's chunk planner outputs (util/mat_size.cu) on the CPU.

    make -C oracle _ref/libref_matsize.so
    python tests/golden/make_planner_golden.py  # writes tests/golden/ref_planner.json

find_mat_size_syrk / find_mat_size_trsm are plain host C++; the library is
loaded with ctypes through their mangled names and the -1-terminated arrays
are recorded for a spread of n.
"""
import ctypes
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))

NS = [1, 2, 100, 1000, 2046, 2048, 2050, 4094, 4096, 5000, 8190, 8192, 8194, 12000, 16384, 16386, 20000, 24576,
      30000, 32768, 40000, 49152, 65536, 70000, 100000]


def run():
    lib = ctypes.CDLL(os.path.join(ROOT, "oracle", "_ref", "libref_matsize.so"))
    out = {}
    for kind in ("syrk", "trsm"):
        fn = getattr(lib, f"_Z18find_mat_size_{kind}lPi")
        fn.restype = ctypes.POINTER(ctypes.c_int64)
        fn.argtypes = [ctypes.c_int64, ctypes.POINTER(ctypes.c_int)]
        res = {}
        for n in NS:
            length = ctypes.c_int(0)
            p = fn(n, ctypes.byref(length))
            vals = []
            i = 0
            while p[i] != -1:
                vals.append(int(p[i]))
                i += 1
            res[str(n)] = {"chunks": vals, "length": length.value}
        out[kind] = res
    return out


if __name__ == "__main__":
    with open(os.path.join(HERE, "ref_planner.json"), "w") as f:
        json.dump(run(), f, indent=1, sort_keys=True)
    print("wrote ref_planner.json")
