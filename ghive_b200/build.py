"""Builds the CUDA library libghive_b200.so in-tree for sm_100a.

    python -m ghive_b200.build [--jobs N] [--verbose]

Every .cu under ghive_b200/csrc is compiled with nvcc for
`-gencode arch=compute_100a,code=sm_100a` and linked into
ghive_b200/lib/libghive_b200.so (the library the Python layer, the tests and
the benchmark load).  Objects are rebuilt only when a source or header is
newer than them.
"""
import argparse
import concurrent.futures as cf
import glob
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIBDIR, "libghive_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-O3", "-I" + os.path.join(ROOT, "include")]


def nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _headers():
    return glob.glob(os.path.join(CSRC, "**", "*.cuh"), recursive=True) + \
        glob.glob(os.path.join(CSRC, "**", "*.hpp"), recursive=True) + \
        [os.path.join(ROOT, "include", "ghive_b200.h")]


def _stale(obj, src, hdr_mtime):
    if not os.path.exists(obj):
        return True
    m = os.path.getmtime(obj)
    return m < os.path.getmtime(src) or m < hdr_mtime


# Headers the run-time compiler (NVRTC) needs for the specialised group-by
# kernels, embedded in the library under the names their #includes use.
JIT_HEADERS = [("ghb_gb_sig.cuh", os.path.join(CSRC, "ghb_gb_sig.cuh")),
               ("ghb_groupby.cuh", os.path.join(CSRC, "ghb_groupby.cuh")),
               ("ghb_internal.cuh", os.path.join(CSRC, "ghb_internal.cuh")),
               ("../../include/ghive_b200.h", os.path.join(ROOT, "include", "ghive_b200.h"))]


def _jit_headers_source(path):
    """Writes a C++ file defining the embedded header table (when stale)."""
    newest = max(os.path.getmtime(f) for _, f in JIT_HEADERS)
    if os.path.exists(path) and os.path.getmtime(path) >= newest:
        return path
    out = ["// generated by ghive_b200/build.py: headers for run-time compilation"]
    names, srcs = [], []
    for name, f in JIT_HEADERS:
        text = open(f).read()
        delim = "GHBJIT"
        assert ")" + delim + '"' not in text
        names.append('"%s"' % name)
        srcs.append('R"%s(%s)%s"' % (delim, text, delim))
    out.append("extern const int ghb_jit_nheaders = %d;" % len(JIT_HEADERS))
    out.append("extern const char* const ghb_jit_header_names[] = {%s};" % ", ".join(names))
    out.append("extern const char* const ghb_jit_header_srcs[] = {\n%s};" % ",\n".join(srcs))
    with open(path + ".tmp", "w") as fh:
        fh.write("\n".join(out) + "\n")
    os.replace(path + ".tmp", path)
    return path


def _cuda_lib_dir(cc):
    return os.path.join(os.path.dirname(os.path.dirname(os.path.realpath(cc))), "lib64")


def build(jobs=None, verbose=False, extra_flags=()):
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    srcs.append(_jit_headers_source(os.path.join(BUILD, "ghb_jit_headers.cpp")))
    hdr_mtime = max(os.path.getmtime(h) for h in _headers())
    cc = nvcc()
    objs, todo = [], []
    for s in srcs:
        o = os.path.join(BUILD, os.path.splitext(os.path.basename(s))[0] + ".o")
        objs.append(o)
        if _stale(o, s, hdr_mtime) or extra_flags:
            todo.append((s, o))

    def compile_one(so):
        s, o = so
        cmd = [cc] + ARCH + NVCC_FLAGS + list(extra_flags) + ["-c", s, "-o", o]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s%s" % (s, r.stdout, r.stderr))
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr)
        return o

    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count()) as ex:
        list(ex.map(compile_one, todo))
    if todo or not os.path.exists(LIB):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + \
            ["-lcudart", "-lnvrtc", "-Xlinker", "-rpath," + _cuda_lib_dir(cc)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-info", action="store_true", help="print registers/spills per kernel")
    a = ap.parse_args()
    extra = ("-Xptxas", "-v") if a.ptxas_info else ()
    print(build(a.jobs, a.verbose or a.ptxas_info, extra))
    sys.exit(0)
