"""Scenarios run by the bounds-checked and the ordinary library alike
(tests/test_gpu_bounds.py): every precision on tile shapes with and without
a helper warp, partial tiles, bulk-copy staging and ordinary loads,
reflecting edges, persistent scheduling, linked z-slabs, the WENO3
reconstruction, and the host-resident streamed run (stages launched over
tile ranges, chunks thinner than the stencil's reach)."""
import numpy as np

ABS, REF = 0, 1


def run_cases(mpcf):
    from conftest import cloud_state
    import mpcf.decomp as dc
    out = {}
    dims = (44, 19, 14)
    bc = (ABS, REF, ABS, ABS, REF, ABS)
    U0 = cloud_state(dims, nb=3)
    tilings = [(3, 5, False, False), (7, 9, True, True), (8, 4, True, True), (8, 64, False, True)]
    for prec in ("fp32_ref", "mixed", "fp64"):
        dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
        for tl in tilings + ([(15, 7, False, True)] if prec == "fp32_ref" else []):
            with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
                s.set_tiling(*tl)
                s.set_state([np.asarray(a, dtype=dt) for a in U0])
                s.step(cfl=0.3)
                s.step(cfl=0.3)
                U, R = s.get_state()
                key = f"{prec}_{tl[0]}_{tl[1]}_{int(tl[2])}_{int(tl[3])}"
                out["err_" + key] = np.array([s.error_word()])
                for q in range(7):
                    out[f"U{q}_{key}"] = U[q]
                    out[f"R{q}_{key}"] = R[q]
    for prec, tl in (("fp32", (7, 9, True, True)), ("fp32", (8, 64, False, True)),
                     ("fp64_fast", (7, 9, True, True)), ("fp64_fast", (3, 5, False, False))):
        dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
        with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
            s.set_tiling(*tl)
            s.set_state([np.asarray(a, dtype=dt) for a in U0])
            s.step(cfl=0.3)
            U, R = s.get_state()
            key = f"{prec}_{tl[0]}_{tl[1]}_{int(tl[2])}_{int(tl[3])}"
            out["err_" + key] = np.array([s.error_word()])
            for q in range(7):
                out[f"U{q}_{key}"] = U[q]
                out[f"R{q}_{key}"] = R[q]
    for prec in ("fp32_ref", "fp64"):
        dt = mpcf.dtype_of(mpcf.PRECISIONS[prec])
        with mpcf.Solver([dims], bc=[bc], precision=prec) as s:
            s.set_weno_order(3)
            s.set_tiling(7, 9, True, True)
            s.set_state([np.asarray(a, dtype=dt) for a in U0])
            s.step(cfl=0.3)
            U, R = s.get_state()
            out[f"err_weno3_{prec}"] = np.array([s.error_word()])
            for q in range(7):
                out[f"U{q}_weno3_{prec}"] = U[q]
    # streamed run: 7 two-plane layers in 7 chunks, a stage of a chunk
    # waiting for the two chunks above it
    with mpcf.Solver([dims], bc=[bc], precision="mixed") as s:
        s.set_tiling(8, 2, True, True)
        host = [np.array(a, dtype=np.float32) for a in U0]
        s.run_host(host, 2, cfl=0.3, nchunks=7)
        out["err_streamed"] = np.array([s.error_word()])
        for q in range(7):
            out[f"U{q}_streamed"] = host[q]
    gdims = (40, 24, 30)
    s, ext = dc.slab_solver(gdims, 3, bc=bc, precision="mixed")
    with s:
        s.set_tiling(8, 5, True, True)
        dc.scatter_state(s, gdims, ext, cloud_state(gdims, nb=3))
        s.run(2, cfl=0.3, graph=True)
        U, R = dc.gather_state(s, ext)
        out["err_slabs"] = np.array([s.error_word()])
        for q in range(7):
            out[f"U{q}_slabs"] = U[q]
            out[f"R{q}_slabs"] = R[q]
    return out
