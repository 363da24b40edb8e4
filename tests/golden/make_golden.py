"""Generate the golden vectors in tests/golden/ from the reference solver itself.

Runs the reference (hellojxt/PPPM-TDBEM compiled from its own sources into
oracle/_ref/libpppm_ref.so by oracle/Makefile) on a CUDA device and stores its outputs as
compressed .npz fixtures:

  tdbem.npz          lambda and the 16 wave numbers (bem.h:264-277) for two (dt, h)
  pairs.npz          single-pair TDBEM weights (face->point, regular / edge / vertex /
                     identical face->face) evaluated by the reference's device code
  fdtd.npz           impulse propagation with the absorbing boundary, 40 steps, res 16
  pml.npz            the same with a 3-layer PML
  sphere_small.npz   icosphere subdivision 2 at res 24: triangles, lists, GridCache and
                     FaceCache records, interpolation weights, listener series (300 steps)
  static_sphere.npz  the 1280-triangle sphere at res 32: listener series over 2000 steps,
                     list sizes and non-empty cells
  moving_small.npz   moving subdivision-2 sphere at res 24 with a mesh update every 10
                     steps: listener series and lists after the last update
  cells.npz          cell labels, nearest triangles and ghost indices before and after a move,
                     and the fresh-cell fill of grid slots t and t-1

Usage (on a machine with a GPU and oracle/_ref built):
    python tests/golden/make_golden.py OUTDIR            # every fixture but noise.npz
    python tests/golden/make_golden.py OUTDIR --noise    # noise.npz: repeats of three scenes
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "pppm-tdbem_b200", "python"))

from oracle import oracle as O  # noqa: E402
from pppm_b200 import scenes  # noqa: E402


def sphere_small_scene(res=24, sub=2, radius=0.1):
    v, f = scenes.icosphere(sub)
    v = (v * radius).astype(np.float32)
    h, mn = scenes.grid_for_bbox(v.min(0), v.max(0), res, 2.0)
    dt = np.float32(0.5 * h / (np.sqrt(3) * 340.3))
    return v, f, h, mn, dt


def moving_small_verts(v0, step, dt):
    t = step * float(dt)
    R = scenes.rotation_matrix([0.3, 0.5, 0.8], 40.0 * t)
    v = v0.astype(np.float64) @ R.T
    v[:, 0] += 0.01 * np.sin(2 * np.pi * 60.0 * t)
    return v.astype(np.float32)


def main(out):
    os.makedirs(out, exist_ok=True)
    rng = np.random.default_rng(2024)

    # ---- TDBEM constants
    cases = [(1.0603700e-05, 0.0125), (1.3612e-05, 0.0086)]
    lam, wave = [], []
    for dt, h in cases:
        l, w = O.reference_tdbem(dt, h)
        lam.append(l)
        wave.append(w)
    np.savez_compressed(os.path.join(out, "tdbem.npz"), cases=np.array(cases), lam=np.array(lam), wave=np.array(wave))

    # ---- single-pair weights
    dt, h = 1.0603700e-05, 0.0125
    V = np.array([[0, 0, 0], [0.01, 0, 0], [0, 0.012, 0], [0.011, 0.009, 0.003], [-0.004, 0.006, 0.008],
                  [0.03, 0.02, -0.01], [0.035, 0.028, -0.012], [0.029, 0.031, -0.004]], np.float32)
    pairs = [("point", [0, 1, 2], None, [0.02, 0.01, 0.015]),
             ("point", [0, 1, 2], None, [0.004, 0.004, 0.001]),
             ("regular", [5, 6, 7], [0, 1, 2], None),
             ("identical", [0, 1, 2], [0, 1, 2], None),
             ("edge", [0, 1, 2], [1, 3, 2], None),
             ("vertex", [0, 1, 2], [0, 4, 5], None)]
    kinds, srcs, dsts, pts, ws = [], [], [], [], []
    for kind, src, dst, pt in pairs:
        if kind == "point":
            w = O.reference_weight(dt, h, V, src, point=pt)
        else:
            w = O.reference_weight(dt, h, V, src, face=dst)
        kinds.append(kind)
        srcs.append(src)
        dsts.append(dst if dst is not None else [-1, -1, -1])
        pts.append(pt if pt is not None else [0, 0, 0])
        ws.append(w)
    np.savez_compressed(os.path.join(out, "pairs.npz"), dt=dt, h=h, verts=V, kinds=np.array(kinds), src=np.array(srcs),
                        dst=np.array(dsts), pts=np.array(pts, np.float32), w=np.array(ws))

    # ---- bare FDTD with ABC and with PML
    for name, pml in (("fdtd", 0), ("pml", 3)):
        res, dl, dtf = 16, 0.01, np.float32(0.5 * 0.01 / (np.sqrt(3) * 340.3))
        f = O.ReferenceFDTD(res, dl, dtf, pml)
        g0 = np.zeros((res,) * 3, np.float32)
        g0[8, 8, 8] = 1.0
        g0[5:11, 6:10, 7:9] += rng.uniform(-0.1, 0.1, size=(6, 4, 2)).astype(np.float32)
        f.step(1)  # t: -1 -> 0 with zero fields
        f.write(0, g0)
        f.write(-1, 0.5 * g0)
        init_t, init_tm1 = f.grid(0).copy(), f.grid(-1).copy()
        f.step(40)
        np.savez_compressed(os.path.join(out, name + ".npz"), res=res, dl=dl, dt=dtf, pml=pml, init_t=init_t,
                            init_tm1=init_tm1, t=f.t, grid_t=f.grid(0), grid_tm1=f.grid(-1), grid_tm2=f.grid(-2))
        f.close()

    # ---- small static sphere: tables, lists, listener
    v, fc, h, mn, dts = sphere_small_scene()
    res = 24
    r = O.Reference(res, h, dts, mn)
    r.set_mesh(v, fc)
    geom, cells = r.triangles()
    L = r.lists()
    gc = r.grid_cache()
    interp = r.interp()
    # face pairs = (centre, neighbour) over every centre's 4^3 list
    pairs = []
    b4 = L["b4_cells"]
    bl = L["b4_tris"]
    n4 = L["n4_tris"]
    ob = on = 0
    cnt4 = []
    for x, y, z, nb in b4:
        centres = bl[ob: ob + nb]
        ob += nb
        # 4^3 list length of this base cell from the cell counts
        cc = L["cell_counts"].reshape((res,) * 3)
        ln = int(cc[max(x - 1, 0): x + 3, max(y - 1, 0): y + 3, max(z - 1, 0): z + 3].sum())
        lst = n4[on: on + ln]
        on += ln
        cnt4.append(ln)
        for c in centres:
            for j in lst:
                pairs.append((c, j))
    pairs = np.array(pairs, np.int32)
    fr = r.face_cache(pairs)
    steps = 300
    acc = np.repeat(np.sin(2 * np.pi * 1500.0 * np.arange(steps) * float(dts)).astype(np.float32)[:, None], len(fc), 1)
    listeners = [(20, 20, 20), (12, 12, 17)]
    series = r.run(acc, listeners)
    np.savez_compressed(os.path.join(out, "sphere_small.npz"), verts=v, tris=fc, h=h, min_pos=mn, dt=dts, res=res,
                        geom=geom, cells=cells, n3_cells=L["n3_cells"], n3_tris=L["n3_tris"], b4_cells=b4,
                        b4_tris=bl, n4_tris=n4, n4_len=np.array(cnt4, np.int32), cell_counts=L["cell_counts"],
                        grid_cache=gc.view(np.uint8), face_pairs=pairs, face_cache=fr.view(np.uint8), interp=interp,
                        acc_freq=1500.0, steps=steps, listeners=np.array(listeners), series=series,
                        final_grid=r.grid(0))
    r.close()

    # ---- the 1280-triangle static sphere (res 32, 2000 steps)
    sc = scenes.StaticSphere()
    r = O.Reference(sc.res, sc.h, sc.dt, sc.min_pos)
    r.set_mesh(sc.verts, sc.tris)
    L = r.lists()
    series = r.run(sc.acc(0, sc.steps), [sc.listener])
    np.savez_compressed(os.path.join(out, "static_sphere.npz"), series=series, n3_cells=L["n3_cells"],
                        cell_counts=L["cell_counts"], sizes=np.array([len(L["n3_cells"]), len(L["n3_tris"]),
                                                                      len(L["b4_cells"]), len(L["n4_tris"])]))
    r.close()

    # ---- small moving sphere
    v0, fc, h, mn, dts = sphere_small_scene()
    r = O.Reference(res, h, dts, mn)
    r.set_mesh(moving_small_verts(v0, 0, dts), fc)
    steps, every = 200, 10
    acc = np.repeat(np.sin(2 * np.pi * 1200.0 * np.arange(steps) * float(dts)).astype(np.float32)[:, None], len(fc), 1)
    series = []
    for s0 in range(0, steps, every):
        if s0 > 0:
            r.update_mesh(moving_small_verts(v0, s0, dts))
        series.append(r.run(acc[s0: s0 + every], [(20, 20, 20)]))
    L = r.lists()
    np.savez_compressed(os.path.join(out, "moving_small.npz"), v0=v0, tris=fc, h=h, min_pos=mn, dt=dts, res=res,
                        steps=steps, every=every, series=np.concatenate(series), n3_cells=L["n3_cells"],
                        n3_tris=L["n3_tris"], cell_counts=L["cell_counts"])
    r.close()

    # ---- cell labels and fresh cells
    v0, fc, h, mn, dts = sphere_small_scene()
    c = O.ReferenceCells(res, h, dts, mn)
    acc0 = rng.uniform(-1, 1, len(fc)).astype(np.float32)
    c.set_mesh(v0, fc, acc0)
    before = c.read()
    g_t = rng.uniform(-1, 1, (res,) * 3).astype(np.float32)
    g_tm1 = rng.uniform(-1, 1, (res,) * 3).astype(np.float32)
    c.write_grid(0, g_t)
    c.write_grid(-1, g_tm1)
    v1 = v0.copy()
    v1[:, 0] += 1.3 * h  # rigid shift: cells behind the sphere turn from SOLID to AIR
    acc1 = rng.uniform(-1, 1, len(fc)).astype(np.float32)
    c.update_mesh(v1, acc1)
    after = c.read()
    np.savez_compressed(os.path.join(out, "cells.npz"), v0=v0, v1=v1, tris=fc, h=h, min_pos=mn, dt=dts, res=res,
                        acc0=acc0, acc1=acc1, g_t=g_t, g_tm1=g_tm1, type0=before["type"], nearest0=before["nearest"],
                        ghost0=before["ghost"], type1=after["type"], nearest1=after["nearest"], ghost1=after["ghost"],
                        reflect1=after["reflect"], out_t=c.grid(0), out_tm1=c.grid(-1))
    c.close()
    print("golden vectors written to", out)


def noise_floor(out, repeats=3):
    """The reference's own run-to-run spread: the same inputs run several times (its float
    atomics sum in a different order each run).  noise.npz: series of each repeat for the
    static sphere (2000 steps), the small sphere (300 steps) and the benchmarked moving scene
    (res 64, 8820 steps in 128 motion frames)."""
    os.makedirs(out, exist_ok=True)
    sc = scenes.StaticSphere()
    big = []
    for _ in range(repeats):
        r = O.Reference(sc.res, sc.h, sc.dt, sc.min_pos)
        r.set_mesh(sc.verts, sc.tris)
        big.append(r.run(sc.acc(0, sc.steps), [sc.listener])[:, 0])
        r.close()
    v, fc, h, mn, dts = sphere_small_scene()
    acc = np.repeat(np.sin(2 * np.pi * 1500.0 * np.arange(300) * float(dts)).astype(np.float32)[:, None], len(fc), 1)
    small = []
    for _ in range(repeats):
        r = O.Reference(24, h, dts, mn)
        r.set_mesh(v, fc)
        small.append(r.run(acc, [(20, 20, 20)])[:, 0])
        r.close()
    # the benchmarked moving scene (res 64, 5120 + 1280 triangles), its whole 8820-step run
    ms = scenes.MovingScene()
    nframes = ms.frame_of_step(ms.steps - 1) + 1
    ranges = scenes.frame_ranges(ms, nframes - 1)
    ranges[-1] = (ranges[-1][0], ms.steps)
    acc = ms.acc(0, ms.steps)
    moving = []
    for _ in range(repeats):
        r = O.Reference(ms.res, ms.h, ms.dt, ms.min_pos)
        r.set_mesh(ms.frame_verts(0), ms.tris)
        run = []
        for f, (a, b) in enumerate(ranges):
            if f:
                r.update_mesh(ms.frame_verts(f))
            run.append(r.run(acc[a:b], [ms.listener])[:, 0])
        moving.append(np.concatenate(run))
        r.close()
    np.savez_compressed(os.path.join(out, "noise.npz"), static_sphere=np.array(big), sphere_small=np.array(small),
                        moving64=np.array(moving))
    print("noise floor written to", out)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args:
        sys.exit("usage: make_golden.py OUTDIR [--noise]  (then copy the .npz files into tests/golden/)")
    out = args[0]
    if "--noise" in sys.argv:
        noise_floor(out)
    else:
        main(out)
