"""Builds the solver library and command-line tools in-tree (dds_gpu_b200/_lib/).

    python -m dds_gpu_b200.build            # libddg.so, libddg_check.so, dd_gpu, dd_stream
    python -m dds_gpu_b200.build --force    # rebuild even when up to date

nvcc compiles for sm_100a only (-gencode arch=compute_100a,code=sm_100a); the output
travels with the source tree, so a machine with the same image needs no rebuild.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "_lib")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(LIB_DIR, "libddg.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-I" + INCLUDE, "-I" + CSRC]

# target -> (sources, extra flags, kind)
TARGETS = {
    "libddg.so": (["ddg_api.cu"], ["-shared"], "lib"),
    # the same library with every stack, TT and task index checked before use (tests)
    "libddg_check.so": (["ddg_api.cu"], ["-shared", "-DDDG_BOUNDS_CHECK"], "lib"),
    # 12-byte signature TT entries (a speed option, not strictly exact)
    "libddg_sig.so": (["ddg_api.cu"], ["-shared", "-DDDG_TT_SIG"], "lib"),
}
CLI = {
    "dd_gpu": "cli_dd_gpu.cpp",
    "dd_stream": "cli_dd_stream.cpp",
}


def _deps():
    files = []
    for d in (CSRC, INCLUDE):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".h", ".hpp", ".cpp")):
                files.append(os.path.join(d, f))
    return files


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd[:3]) + " ...")
    return r.stdout + r.stderr


def build(force=False, verbose=False):
    """Compiles what is out of date; returns the library path."""
    os.makedirs(LIB_DIR, exist_ok=True)
    deps = _deps()
    for name, (srcs, extra, _) in TARGETS.items():
        out = os.path.join(LIB_DIR, name)
        if force or _stale(out, deps):
            tmp = out + ".tmp"
            log = _run([NVCC] + NVFLAGS + extra + (["-Xptxas", "-v"] if verbose else []) +
                       ["-o", tmp] + [os.path.join(CSRC, s) for s in srcs])
            os.replace(tmp, out)
            if verbose:
                print(log)
    for name, src in CLI.items():
        path = os.path.join(CSRC, src)
        if not os.path.exists(path):
            continue
        out = os.path.join(LIB_DIR, name)
        if force or _stale(out, deps):
            tmp = out + ".tmp"
            _run(["g++", "-O2", "-std=c++17", "-pthread", "-I" + INCLUDE, "-I" + CSRC, "-o", tmp, path,
                  "-L" + LIB_DIR, "-lddg", "-Wl,-rpath,$ORIGIN", "-L/usr/local/cuda/lib64", "-lcudart"])
            os.replace(tmp, out)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIB)
