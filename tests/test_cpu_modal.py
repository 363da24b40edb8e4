"""The scene host's Modal objects (the reference's RigidBody, src/utils/RigidBody.cu) on the CPU:
boundary faces of a tet mesh, and the surface accelerations of the modal IIR driven by contact
impulses, exported by `pppm_demo --modal-accs` and checked against a float64 restatement of the
same published recipe (Rayleigh-damped modes, half-sine contact forces of 0.5 ms, face
acceleration = face normal . mean vertex mode shape x modal acceleration).  Tolerance: relative L2
1e-4 over the run (the host computes in float32 as the reference does)."""
import math
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "pppm-tdbem_b200", "bin", "pppm_demo")
ALPHA, BETA = 30.0, 1e-6  # "plastic" (src/utils/material.h)
TAU = 0.0005


def _cube_tets():
    v = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float) * 0.05
    # 5-tet split of the unit cube (corner tets + the central one)
    tets = [[0, 1, 2, 4], [3, 1, 2, 7], [5, 1, 4, 7], [6, 2, 4, 7], [1, 2, 4, 7]]
    return v, np.array(tets)


def _write_object(d, rng):
    v, tets = _cube_tets()
    np.savetxt(os.path.join(d, "vertices.txt"), v, fmt="%.9g")
    np.savetxt(os.path.join(d, "tets.txt"), tets[:, [2, 0, 3, 1]].astype(float), fmt="%.1f")  # unsorted
    freqs = np.array([450.0, 1300.0, 2900.0, 7000.0, 16000.0])  # the last one is above 15 kHz
    lam = (2 * math.pi * freqs) ** 2
    np.savetxt(os.path.join(d, "eigenvalues.txt"), lam, fmt="%.9g")
    vecs = rng.standard_normal((3 * len(v), len(lam)))
    np.savetxt(os.path.join(d, "eigenvectors.txt"), vecs, fmt="%.9g")
    with open(os.path.join(d, "motion.txt"), "w") as f:
        f.write("0 0 0 0 0 0 0 1\n0.001 0.01 0 0 0 0 0 1\n")
    imps = [(0.0020, 3, (0.0, 0.0, 1.0), 2.0), (0.00226, 6, (1.0, 0.0, 0.0), 0.5)]
    with open(os.path.join(d, "contact.txt"), "w") as f:
        for t, vid, n, mag in imps:
            f.write("%.9g %d %g %g %g %g\n" % (t, vid, n[0], n[1], n[2], mag))
    return v, tets, lam[:4], vecs[:, :4], imps


def _boundary_faces(tets):
    count = {}
    for t in tets:
        t = sorted(t)
        for skip in range(4):
            key = tuple(x for i, x in enumerate(t) if i != skip)
            count[key] = count.get(key, 0) + 1
    return {k for k, c in count.items() if c == 1}


@pytest.mark.skipif(not os.path.exists(DEMO), reason="scene host not built")
def test_modal_object_surface_accelerations(tmp_path):
    rng = np.random.default_rng(2)
    d = str(tmp_path / "obj")
    os.makedirs(d)
    v, tets, lam, vecs, imps = _write_object(d, rng)
    rate, n = 44100.0, 240
    out = str(tmp_path / "accs.txt")
    r = subprocess.run([DEMO, "--modal-accs", d, str(rate), str(n), out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    lines = open(out).read().split("\n")
    nf, nm, t0 = lines[0].split()
    nf, nm, t0 = int(nf), int(nm), float(t0)
    faces = np.array([[int(x) for x in lines[1 + i].split()] for i in range(nf)])
    got = np.array([[float(x) for x in lines[1 + nf + s].split()] for s in range(n)])
    assert nm == 4  # modes up to 15 kHz
    # boundary faces: each face of exactly one tet, wound away from that tet's fourth vertex
    assert {tuple(sorted(f)) for f in faces} == _boundary_faces(tets) and nf == 12
    centre = v.mean(0)
    normals = []
    for f in faces:
        a, b, c = v[f]
        nrm = np.cross(b - a, c - a)
        nrm /= np.linalg.norm(nrm)
        assert np.dot(nrm, (a + b + c) / 3 - centre) > 0  # the cube is convex: outward
        normals.append(nrm)
    normals = np.array(normals)

    # float64 restatement
    dt = 1.0 / rate
    omega = np.sqrt(lam)
    ksi = (ALPHA + BETA * lam) / (2 * omega)
    wd = omega * np.sqrt(1 - ksi ** 2)
    eps = np.exp(-ksi * omega * dt)
    theta, gamma = wd * dt, np.arcsin(ksi)
    c1, c2 = 2 * eps * np.cos(theta), -eps ** 2
    c3 = 2 * (eps * np.cos(theta + gamma) - eps ** 2 * np.cos(2 * theta + gamma)) / (3 * omega * wd)
    surf = np.array([[np.dot(vecs[[3 * f[0] + k for k in range(3)], i] / 3 + vecs[[3 * f[1] + k for k in range(3)], i] / 3
                             + vecs[[3 * f[2] + k for k in range(3)], i] / 3, normals[j]) for i in range(4)]
                     for j, f in enumerate(faces)])
    t = 0.0
    while t + dt < imps[0][0]:
        t += dt
    assert abs(t - t0) < 1e-6
    q1 = q2 = q3 = np.zeros(4)
    want = []
    for s in range(n):
        t += dt
        force = np.zeros(4)
        for ti, vid, nrm, mag in imps:
            if t >= ti and t - ti <= TAU:
                j = np.array(nrm) * mag * math.sin(math.pi * (t - ti) / TAU)
                force += vecs[3 * vid: 3 * vid + 3].T @ j
        q0 = c1 * q1 + c2 * q2 + c3 * force
        q1, q2, q3 = q0, q1, q2
        want.append(surf @ ((q1 + q3 - 2 * q2) / dt ** 2))
    want = np.array(want)
    assert np.abs(want).max() > 0
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err < 1e-4, err


@pytest.mark.skipif(not os.path.exists(DEMO), reason="scene host not built")
def test_modal_object_missing_files_fail_cleanly(tmp_path):
    d = str(tmp_path / "empty")
    os.makedirs(d)
    r = subprocess.run([DEMO, "--modal-accs", d, "44100", "10", str(tmp_path / "x.txt")], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "cannot read" in r.stderr
