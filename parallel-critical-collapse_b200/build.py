"""Builds the B200 engine: libpcc_b200.so (CUDA kernels + C ABI, sm_100a) and
libpcc_host.so (the C++ host classes over the C ABI), in-tree.

    python parallel-critical-collapse_b200/build.py [--force]

Each CUDA translation unit is compiled by its own nvcc process (the march
kernel once per Ntau), in parallel; objects are rebuilt when a source or
header is newer.  No JIT cache is involved: the .so files sit next to this
script and travel with the repository checkout.
"""
import argparse
import concurrent.futures as cf
import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
CSRC = PKG / "csrc"
HOST = PKG / "host"
OBJ = PKG / "_build"
LIB = PKG / "libpcc_b200.so"
HOSTLIB = PKG / "libpcc_host.so"
CLI = PKG / "cc_b200"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-I" + str(REPO / "include"),
           "-I" + str(CSRC), "--expt-relaxed-constexpr"] + ARCH
MARCH_NS = [128, 256, 512, 1024, 2048]


def _nvcc():
    for c in [os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"]:
        if c and (Path(c).exists() or c == "nvcc"):
            return c
    return "nvcc"


def _units():
    units = []
    for n in MARCH_NS:
        for pair in (0, 1):
            units.append((CSRC / "march.cu", OBJ / f"march_n{n}_p{pair}.o",
                          [f"-DPCC_MARCH_N={n}", f"-DPCC_MARCH_PAIR={pair}"]))
    units.append((CSRC / "march.cu", OBJ / "march_n1024_p2.o", ["-DPCC_MARCH_N=1024", "-DPCC_MARCH_PAIR=2"]))
    units.append((CSRC / "march.cu", OBJ / "march_dispatch.o", ["-DPCC_MARCH_DISPATCH"]))
    units.append((CSRC / "march.cu", OBJ / "march_batch.o", ["-DPCC_MARCH_BATCH"]))
    for name in ["boundary", "lu", "newton", "pcc_abi", "resample", "serve", "static_scratch"]:
        units.append((CSRC / f"{name}.cu", OBJ / f"{name}.o", []))
    return units


def _newest_dep():
    deps = list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + [REPO / "include" / "pcc.h", Path(__file__)]
    return max(p.stat().st_mtime for p in deps if p.exists())


def _compile(unit, force, verbose):
    src, obj, extra = unit
    dep = max(_newest_dep(), src.stat().st_mtime)
    if not force and obj.exists() and obj.stat().st_mtime >= dep:
        return obj, None
    user = os.environ.get("PCC_NVCC_EXTRA", "").split()  # extra nvcc flags, e.g. -D options
    cmd = [_nvcc()] + NVFLAGS + user + extra + ["-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name} {extra}:\n{r.stderr[-4000:]}")
    return obj, r.stderr if verbose else None


def build_cuda(force=False, verbose=False, jobs=None):
    OBJ.mkdir(exist_ok=True)
    units = _units()
    logs = []
    with cf.ThreadPoolExecutor(max_workers=jobs or min(len(units), os.cpu_count() or 4)) as ex:
        for obj, log in ex.map(lambda u: _compile(u, force, verbose), units):
            if log:
                logs.append(log)
    objs = [str(u[1]) for u in units]
    newest = max(Path(o).stat().st_mtime for o in objs)
    if force or not LIB.exists() or LIB.stat().st_mtime < newest:
        cmd = [_nvcc(), "-shared"] + ARCH + ["-o", str(LIB)] + objs + ["-lcudart"]
        subprocess.run(cmd, check=True)
    return logs


def build_host(force=False):
    srcs = sorted(HOST.glob("*.cpp"))
    if not srcs:
        return
    hdrs = list(HOST.glob("*.hpp")) + [REPO / "include" / "pcc.h"]
    dep = max(p.stat().st_mtime for p in srcs + hdrs + [LIB])
    if not force and HOSTLIB.exists() and HOSTLIB.stat().st_mtime >= dep:
        return
    lib_srcs = [str(s) for s in srcs if s.name != "main.cpp"]
    cxx = "g++"
    import sysconfig

    json_inc = Path(sysconfig.get_paths()["purelib"]) / "include" / "cudnn_frontend" / "thirdparty"  # nlohmann/json
    flags = ["-std=c++17", "-O2", "-fPIC", "-I" + str(REPO / "include"), "-I" + str(HOST), "-I" + str(json_inc)]
    subprocess.run([cxx, "-shared"] + flags + ["-o", str(HOSTLIB)] + lib_srcs +
                   ["-L" + str(PKG), "-l:libpcc_b200.so", "-Wl,-rpath,$ORIGIN", "-lpthread"], check=True)
    main = HOST / "main.cpp"
    if main.exists():
        subprocess.run([cxx] + flags + ["-o", str(CLI), str(main), "-L" + str(PKG), "-l:libpcc_host.so",
                                        "-l:libpcc_b200.so", "-Wl,-rpath,$ORIGIN"], check=True)


def build_oracle(force=False):
    sys.path.insert(0, str(REPO / "oracle"))
    import oracle_lib  # noqa: E402  (test infrastructure: the checker, built beside the product)

    oracle_lib.build(force=force)
    # the compiled reference: oracle/build_ref.sh finds the reference checkout
    # itself and keeps the prebuilt oracle/_ref where there is none
    if force or not (REPO / "oracle" / "_ref" / "libpcc_ref.so").exists():
        subprocess.run(["bash", str(REPO / "oracle" / "build_ref.sh")], check=True)


def build_all(force=False, verbose=False):
    logs = build_cuda(force=force, verbose=verbose)
    build_host(force=force)
    build_oracle(force=force)
    return logs


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true", help="print ptxas register/spill reports")
    a = ap.parse_args()
    for log in build_all(force=a.force, verbose=a.verbose):
        print(log)
    print(f"built {LIB}")
