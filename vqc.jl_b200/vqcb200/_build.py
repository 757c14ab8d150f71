"""Builds libvqcb200.so (the sm_100a engine) in-tree with nvcc.

Each .cu under csrc/ is compiled to an object in parallel, then linked into
vqcb200/libvqcb200.so next to this file.  No GPU is needed to build.
build(debug=True) builds libvqcb200_debug.so instead: the same sources with
VQC_DEBUG_CHECKS (device-side index checks that record and skip an access out
of bounds, read with vqc_debug_status), objects under _build_debug/.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
CSRC = os.path.join(PKG_ROOT, "csrc")
REPO = os.path.dirname(PKG_ROOT)
INCLUDE = os.path.join(REPO, "include")
BUILD = os.path.join(PKG_ROOT, "_build")
LIB = os.path.join(HERE, "libvqcb200.so")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
                "--expt-relaxed-constexpr", "-I", INCLUDE, "-I", CSRC]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _deps_mtime():
    paths = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return max(os.path.getmtime(p) for p in paths)


def _compile(src, extra, build_dir=BUILD):
    obj = os.path.join(build_dir, os.path.basename(src) + ".o")
    hdr_time = max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC) if not f.endswith(".cu"))
    hdr_time = max(hdr_time, max(os.path.getmtime(os.path.join(INCLUDE, f)) for f in os.listdir(INCLUDE)))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time):
        return obj, ""
    cmd = [NVCC] + FLAGS + ["-I", build_dir] + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
    return obj, r.stderr


JIT_HEADERS = [("kJitTileDev", "tile_dev.cuh"), ("kJitTileF32", "tile_f32.cuh")]


def write_jit_sources(build_dir=BUILD):
    """_build/jit_src.inc: the device headers the run-time compiled pass
    kernels include, as C++ raw string literals (rewritten only on change)."""
    out = os.path.join(build_dir, "jit_src.inc")
    parts = ["// generated by vqcb200/_build.py from csrc/ (do not edit)\n"]
    for name, f in JIT_HEADERS:
        text = open(os.path.join(CSRC, f)).read()
        if ")VQCJIT" in text:
            raise RuntimeError("%s contains the raw-string delimiter" % f)
        parts.append('static const char* %s = R"VQCJIT(%s)VQCJIT";\n' % (name, text))
    data = "".join(parts)
    if not os.path.exists(out) or open(out).read() != data:
        with open(out, "w") as fh:
            fh.write(data)


def build(verbose=False, extra=(), debug=False):
    """Compile every csrc/*.cu for sm_100a and link libvqcb200.so (incremental);
    debug=True: libvqcb200_debug.so with the device-side index checks."""
    build_dir = BUILD + "_debug" if debug else BUILD
    lib = LIB.replace(".so", "_debug.so") if debug else LIB
    extra = list(extra) + (["-DVQC_DEBUG_CHECKS"] if debug else [])
    os.makedirs(build_dir, exist_ok=True)
    write_jit_sources(build_dir)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra, build_dir), srcs))
    objs = [o for o, _ in results]
    if verbose:
        for (o, log) in results:
            if log.strip():
                print(log, file=sys.stderr)
    if not os.path.exists(lib) or os.path.getmtime(lib) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-o", lib] + objs + ["-lcudart_static", "-lrt", "-lpthread", "-ldl"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return lib


if __name__ == "__main__":
    print(build(verbose=True, extra=sys.argv[1:]))
