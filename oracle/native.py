"""Compiled per-particle work of the oracle (test infrastructure).

oracle/solid2d_cpu.cpp restates, in C++ with OpenMP threads over particles,
the oracle's per-particle residual and complex-step element tangent of the 2D
solid kind with Hencky elasticity (OracleEngine.local and the tangent passes
of OracleEngine.assemble).  The benchmark's CPU-baseline and reference legs
use it on the batched workload, whose blocks are exactly that case.  The
reference's own CPU path is likewise compiled per-particle kernels (Warp on
the CPU) followed by a SciPy sparse direct solve.  The shape functions,
activation, global assembly, solve and G2P stay in NumPy.

build() compiles it into oracle/_build/ with g++; load() returns None when
the library is absent, and the oracle then runs its NumPy path.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "solid2d_cpu.cpp")
LIB = os.path.join(HERE, "_build", "libgw_oracle_cpu.so")
_lib = None


def build(force=False):
    """g++ -O3 -fopenmp into oracle/_build/ (when missing or older than the source)."""
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = LIB + ".tmp"
    subprocess.run(["g++", "-O3", "-fopenmp", "-shared", "-fPIC", "-o", tmp, SRC], check=True,
                   capture_output=True, text=True)
    os.replace(tmp, LIB)
    return LIB


def load():
    """The compiled library, or None when it has not been built."""
    global _lib
    if _lib is None and os.path.exists(LIB):
        lib = C.CDLL(LIB)
        f = lib.gw_oracle_solid2d_hencky
        f.restype = C.c_int
        f.argtypes = [C.c_int64] + [C.c_void_p] * 7 + [C.c_double] * 4 + [C.c_void_p, C.c_int32, C.c_int32] + \
            [C.c_void_p] * 5
        t = lib.gw_oracle_triplets
        t.restype = C.c_int
        t.argtypes = [C.c_int64] + [C.c_void_p] * 4 + [C.c_int32] + [C.c_void_p] * 3
        _lib = lib
    return _lib


def supports(o):
    """Whether engine o's load step is the compiled case: the 2D solid kind
    with Hencky elasticity and no penalty footing."""
    return (o.kind == "solid2d" and o.mat.get("material_name") == "Hencky elasticity"
            and "penalty_factor" not in o.load and load() is not None)


def _ptr(a):
    return C.c_void_p(a.ctypes.data)


def solid2d_local(o, geo, Un, Uo, step, n_steps, want_K):
    """The compiled counterpart of o.local(Un, Uo, geo, step, n_steps,
    want_aux=True) plus, with want_K, the element tangents K[N, 9, 2, 9, 2]
    = -dr/du that the complex-step passes of OracleEngine.assemble form.
    Returns (r[N, 9, 2], K or None, aux)."""
    lower, span, W, Gr, Wa, ids, valid = geo
    N = o.N
    ramp = (step + 1.0) / n_steps
    gy = -o.load.get("gravity_mag", 0.0) * (ramp if o.load.get("gravity_ramp", True) else 1.0)
    fext = np.zeros((N, 2))
    pl = [o.load.get(k, 0.0) for k in ("point_load_value_x", "point_load_value_y")]
    fext[o.ext_flag] = np.array(pl) * ramp
    cont = [np.ascontiguousarray(a, dtype=np.float64) for a in (W, Gr, Un, Uo, o.F_old, o.b_old, o.E, fext)]
    r = np.empty((N, 9, 2))
    K = np.empty((N, 9, 2, 9, 2)) if want_K else None
    F_new, b_new, sigma = np.empty((N, 3, 3)), np.empty((N, 3, 3)), np.empty((N, 3, 3))
    rc = load().gw_oracle_solid2d_hencky(N, *[_ptr(a) for a in cont[:7]], float(o.nu), float(o.p_vol),
                                         float(o.p_rho), float(gy), _ptr(cont[7]), int(bool(want_K)),
                                         int(max(1, o.threads)), _ptr(r), _ptr(K) if want_K else None, _ptr(F_new),
                                         _ptr(b_new), _ptr(sigma))
    if rc != 0:
        raise RuntimeError("gw_oracle_solid2d_hencky: bad arguments")
    return r, K, dict(F_new=F_new, b_new=b_new, sigma=sigma, pi_new=o.pi_new, force=0.0)


def triplets(o, dofs, okd, K):
    """(rows, cols, vals) of the Jacobian entries whose row and column DOFs
    are both free, from the element tangents K[N, 9, 2, 9, 2]: the entries
    and order of the oracle's NumPy masks, listed by the compiled library."""
    N = dofs.shape[0]
    d = np.ascontiguousarray(dofs.reshape(N, 18), dtype=np.int64)
    ok = np.ascontiguousarray(okd.reshape(N, 18), dtype=np.uint8)
    cnt = ok.sum(1, dtype=np.int64) ** 2
    offsets = np.zeros(N, dtype=np.int64)
    np.cumsum(cnt[:-1], out=offsets[1:])
    total = int(cnt.sum())
    rows, cols, vals = np.empty(total, np.int64), np.empty(total, np.int64), np.empty(total)
    rc = load().gw_oracle_triplets(N, _ptr(d), _ptr(ok), _ptr(np.ascontiguousarray(K)), _ptr(offsets),
                                   int(max(1, o.threads)), _ptr(rows), _ptr(cols), _ptr(vals))
    if rc != 0:
        raise RuntimeError("gw_oracle_triplets: bad arguments")
    return rows, cols, vals
