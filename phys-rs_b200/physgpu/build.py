"""Builds libphysgpu.so in-tree with nvcc for sm_100a.

Each translation unit under phys-rs_b200/csrc is compiled to an object file in
phys-rs_b200/_build (rebuilt when it or any header is newer), then linked into
phys-rs_b200/lib/libphysgpu.so.
"""
import concurrent.futures
import glob
import os
import shutil
import subprocess

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REPO = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libphysgpu.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-Wall",
              "--expt-relaxed-constexpr", "-I", os.path.join(REPO, "include")]


def nvcc():
    p = shutil.which("nvcc")
    if p:
        return p
    p = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(p):
        return p
    raise RuntimeError("nvcc not found")


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def build(verbose=False, ptxas_verbose=False, jobs=None):
    """Compile every .cu for sm_100a and link the shared library.  Returns the
    path of libphysgpu.so."""
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(REPO, "include", "*.h"))
    hdr_time = _newest(headers)
    cc = nvcc()
    flags = ARCH + NVCC_FLAGS + (["-Xptxas", "-v"] if ptxas_verbose else [])

    def compile_one(src):
        obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
        if (not ptxas_verbose and os.path.exists(obj)
                and os.path.getmtime(obj) >= max(os.path.getmtime(src), hdr_time)):
            return obj, ""
        cmd = [cc] + flags + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
        return obj, r.stderr

    with concurrent.futures.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        results = list(ex.map(compile_one, sources))
    objs = [o for o, _ in results]
    if verbose or ptxas_verbose:
        for _, log in results:
            if log:
                print(log)
    if (not os.path.exists(LIB)) or os.path.getmtime(LIB) < _newest(objs):
        cmd = [cc] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return LIB


if __name__ == "__main__":
    import sys
    print(build(verbose=True, ptxas_verbose="-v" in sys.argv))
