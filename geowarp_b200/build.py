"""Build the in-tree CUDA library libgeowarp_b200.so for sm_100a.

The library is four translation units (csrc/gw_abi*.cu) compiled in parallel
as relocatable device code (their device status word and index-guard record
are shared) and linked into one shared object next to this file, so it
travels with the source tree.  ``build()`` rebuilds only when a source is
newer than the .so.
"""
import os
import shutil
import subprocess
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libgeowarp_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC", "-rdc=true"]
UNITS = ["gw_abi.cu", "gw_abi_solve.cu", "gw_abi_assemble.cu", "gw_abi_adjoint.cu"]


def _sources():
    out = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cu", ".cuh"))]
    out.append(os.path.join(INCLUDE, "geowarp_b200.h"))
    return out


def needs_build(lib=LIB):
    if not os.path.exists(lib):
        return True
    t = os.path.getmtime(lib)
    return any(os.path.getmtime(s) > t for s in _sources())


def nvcc_path():
    p = shutil.which("nvcc")
    if p:
        return p
    cand = "/usr/local/cuda/bin/nvcc"
    if os.path.exists(cand):
        return cand
    raise RuntimeError("nvcc not found: the geowarp_b200 CUDA library cannot be built")


def build(force=False, verbose=False, extra_flags=(), out=None):
    """Compile the translation units (in parallel) and link libgeowarp_b200.so."""
    out = out or LIB
    if not force and out == LIB and not needs_build():
        return out
    nvcc = nvcc_path()
    with tempfile.TemporaryDirectory(prefix="gw_build_") as tmp:
        procs = []
        for u in UNITS:
            obj = os.path.join(tmp, u.replace(".cu", ".o"))
            cmd = [nvcc, *NVCC_FLAGS, *extra_flags, "-c", "-o", obj, os.path.join(CSRC, u)]
            procs.append((u, obj, subprocess.Popen(cmd, cwd=CSRC, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                                   text=True)))
        log = []
        failed = []
        for u, obj, p in procs:
            so, se = p.communicate()
            log.append(so + se)
            if p.returncode != 0:
                failed.append(f"{u}:\n{so}{se}")
        if failed:
            raise RuntimeError("nvcc failed:\n" + "\n".join(failed))
        part = out + ".tmp"
        cmd = [nvcc, *ARCH, "-rdc=true", "-shared", "-Xcompiler", "-fPIC", "-o", part,
               *[obj for _, obj, _ in procs]]
        res = subprocess.run(cmd, cwd=CSRC, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError("nvcc link failed:\n" + res.stdout + res.stderr)
        if verbose:
            print("".join(log) + res.stdout + res.stderr)
    os.replace(part, out)
    return out


if __name__ == "__main__":
    import sys
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
