"""Generate the golden vectors in tests/golden/seldon_golden.npz by running
the REFERENCE itself (oracle/_ref/libseldon_ref.so, Seldon's own templates
compiled from its headers by oracle/Makefile).

The reference's own test-suite pins no SpMV or solver result, so these
vectors are the pin: the restatement in oracle/seldon_oracle.c must reproduce
every array bit for bit (tests/test_oracle_pin.py).

Run from the repository root after `make -C oracle`:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.pyoracle import Reference  # noqa: E402
from seldon_b200 import matgen  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "seldon_golden.npz")


def main():
    R = Reference()
    rng = np.random.default_rng(20240611)
    g = {}

    def put(prefix, **kw):
        for k, v in kw.items():
            g[f"{prefix}/{k}"] = np.asarray(v)

    mats = {
        "lap2d_9": (matgen.lap2d(9), 81, 81),
        "conv_4": (matgen.convdiff3d(4), 64, 64),
        "rand_37x29": (matgen.random_csr(37, 29, 0.15, seed=5, empty_rows=0.1), 37, 29),
    }
    for name, ((ptr, ind, val), m, n) in mats.items():
        put(f"mat/{name}", ptr=ptr, ind=ind, val=val, m=m, n=n)
        x = rng.standard_normal(n)
        y = rng.standard_normal(m)
        put(f"mltadd/{name}", x=x, y=y, alpha=1.7, beta=-0.3,
            out=R.mltadd(m, n, ptr, ind, val, 1.7, x, -0.3, y))
        xt = rng.standard_normal(m)
        yt = rng.standard_normal(n)
        put(f"mltadd_t/{name}", x=xt, y=yt, alpha=0.9, beta=2.0,
            out=R.mltadd(m, n, ptr, ind, val, 0.9, xt, 2.0, yt, trans=True))

    ptr, ind, val = matgen.lap2d(9)
    up = matgen.upper(ptr, ind, val)
    put("mat/lap2d_9_upper", ptr=up[0], ind=up[1], val=up[2], m=81, n=81)
    x = rng.standard_normal(81)
    y = rng.standard_normal(81)
    put("mltadd_sym/lap2d_9", x=x, y=y, alpha=1.1, beta=0.5,
        out=R.mltadd(81, 81, *up, 1.1, x, 0.5, y, sym=True))

    for t in (0, 2, 3):
        for sym in (0, 1):
            A = up if sym else (ptr, ind, val)
            x0 = rng.standard_normal(81)
            b = rng.standard_normal(81)
            put(f"sor/t{t}_s{sym}", x0=x0, b=b, omega=1.3, it=2,
                out=R.sor(*A, x0, b, 1.3, 2, t, sym=bool(sym)))

    cases = [
        ("cg", "lap2d_9", 0, 0), ("cg", "lap2d_9", 1, 0), ("cg", "lap2d_9", 2, 0),
        ("cg", "lap2d_9", 0, 1), ("cg", "lap2d_9", 2, 1),
        ("bicgstab", "conv_4", 0, 0), ("bicgstab", "conv_4", 1, 0), ("bicgstab", "conv_4", 2, 0),
        ("gmres", "conv_4", 0, 0), ("gmres", "conv_4", 1, 0), ("gmres", "conv_4", 2, 0),
        ("gmres", "lap2d_9", 1, 1),
    ]
    for which, mname, pc, sym in cases:
        (p, i_, v), m, _ = mats[mname]
        A = matgen.upper(p, i_, v) if sym else (p, i_, v)
        xs = rng.uniform(-1, 1, m)
        b = matgen.matvec(p, i_, v, xs)
        xout, code, nb = R.solve(which, *A, b, sym=bool(sym), precond=pc, tol=1e-10,
                                 max_iter=400, restart=6, omega=1.2)
        put(f"solve/{which}_{mname}_p{pc}_s{sym}", b=b, x=xout, code=code, nb=nb,
            tol=1e-10, max_iter=400, restart=6, omega=1.2)

    rot = []
    for a, b in [(3.0, 4.0), (-3.0, 4.0), (4.0, -3.0), (0.0, 0.0), (0.0, 2.0), (2.0, 0.0),
                 (-1e-300, 1e-300), (1.0, -1.0)]:
        rot.append([a, b, *R.genrot(a, b)])
    put("genrot", table=np.array(rot))

    # coordinate -> CSR assembly (ConvertMatrix_from_Coordinates)
    crng = np.random.default_rng(7)
    coo_cases = {
        "gen_dup_i1": (crng.integers(1, 31, 700), crng.integers(1, 23, 700), 1, 0, 0, 0),
        "gen_min": (crng.integers(0, 12, 90), crng.integers(0, 9, 90), 0, 20, 15, 0),
        "sym_both": (crng.integers(0, 40, 500), crng.integers(0, 40, 500), 0, 0, 0, 1),
        "sym_i1_min": (crng.integers(1, 17, 200), crng.integers(1, 17, 200), 1, 30, 30, 1),
        "empty_gen": (np.zeros(0, np.int32), np.zeros(0, np.int32), 0, 6, 4, 0),
        "empty_sym": (np.zeros(0, np.int32), np.zeros(0, np.int32), 0, 6, 6, 1),
    }
    for name, (r, c, index, m_min, n_min, sym) in coo_cases.items():
        v = crng.standard_normal(r.size)
        m, n, op, oi, ov = R.coo_to_csr(r, c, v, index, m_min, n_min, bool(sym))
        put(f"coo/{name}", row=r.astype(np.int32), col=c.astype(np.int32), val=v, index=index,
            m_min=m_min, n_min=n_min, sym=sym, m=m, n=n, ptr=op, ind=oi, out=ov)
    # ILUT: Seldon's own factor (GetIlut) and its Solve / TransSolve
    irng = np.random.default_rng(13)
    ilut_cases = {
        "conv5_ilut": (matgen.convdiff3d(5), False, None, dict(droptol=1e-3)),
        "conv5_perm_piv": (matgen.convdiff3d(5), False, irng.permutation(125),
                           dict(droptol=1e-4, permtol=0.5)),
        "conv5_ilu0": (matgen.convdiff3d(5), False, None, dict(type_ilu=R.ILU_0)),
        "conv5_iluk2": (matgen.convdiff3d(5), False, None, dict(type_ilu=R.ILU_K, fill_level=2)),
        "lap9_sym": (matgen.upper(*matgen.lap2d(9)), True, None, dict(droptol=1e-3)),
    }
    for name, ((p, i_, v), sym, perm, kw) in ilut_cases.items():
        fptr, find, fval, prow, pcol = R.ilut_factor(p, i_, v, sym=sym, perm=perm, **kw)
        n = p.size - 1
        r = irng.standard_normal(n)
        put(f"ilut/{name}", fptr=fptr, find=find, fval=fval, prow=prow, pcol=pcol, sym=int(sym),
            r=r, z=R.ilut_solve(r), zt=R.ilut_solve(r, trans=True))
    np.savez_compressed(OUT, **g)
    print(f"wrote {OUT}: {len(g)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
