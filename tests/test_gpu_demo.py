"""The scene host `pppm_demo CONFIG` end to end on the B200: the reference's config layout, an Audio
object (mesh.obj, motion.txt, accs.txt) beside a Modal object (tet mesh, contact impulses,
eigenmodes), result.txt in the reference's format: the frame rate on line 0, then one sample per
step, with the steps before the Modal object's first contact left silent (zero) at the front."""
import math
import os
import subprocess

import numpy as np
import pytest

from pppm_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "pppm-tdbem_b200", "bin", "pppm_demo")


def _audio(d):
    os.makedirs(d)
    v, f = scenes.icosphere(1)
    v = v * 0.05
    with open(os.path.join(d, "mesh.obj"), "w") as fo:
        for p in v:
            fo.write("v %.7f %.7f %.7f\n" % tuple(p))
        for t in f:
            fo.write("f %d %d %d\n" % tuple(t + 1))
    with open(os.path.join(d, "motion.txt"), "w") as fo:
        fo.write("0 0 0 0 0 0 0 1\n0.001 0 0.002 0 0 0 0 1\n")
    a = np.sin(2 * math.pi * 1500.0 * np.arange(441) / 44100.0)
    np.savetxt(os.path.join(d, "accs.txt"), a, fmt="%.7f")


def _modal(d, rng):
    os.makedirs(d)
    v = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float) * 0.05
    tets = np.array([[0, 1, 2, 4], [3, 1, 2, 7], [5, 1, 4, 7], [6, 2, 4, 7], [1, 2, 4, 7]])
    np.savetxt(os.path.join(d, "vertices.txt"), v, fmt="%.7g")
    np.savetxt(os.path.join(d, "tets.txt"), tets.astype(float), fmt="%.1f")
    lam = (2 * math.pi * np.array([800.0, 2100.0, 5200.0])) ** 2
    np.savetxt(os.path.join(d, "eigenvalues.txt"), lam, fmt="%.9g")
    np.savetxt(os.path.join(d, "eigenvectors.txt"), rng.standard_normal((24, 3)), fmt="%.7g")
    with open(os.path.join(d, "motion.txt"), "w") as fo:
        fo.write("0 0.1 -0.025 -0.025 0 0 0 1\n")
    with open(os.path.join(d, "contact.txt"), "w") as fo:
        fo.write("0.002 7 0 0 1 3.0\n0.0024 0 1 0 0 1.0\n")


def test_demo_audio_and_modal_scene(gpu, tmp_path):
    if not os.path.exists(DEMO):
        pytest.skip("scene host not built")
    rng = np.random.default_rng(5)
    scene = tmp_path / "scene"
    _audio(str(scene / "sphere"))
    _modal(str(scene / "cube"), rng)
    out = tmp_path / "out"
    cfg = tmp_path / "scene.cfg"
    cfg.write_text("{\n"
                   '    inputDir: "%s",\n'
                   '    outputDir: "%s",\n'
                   "    res: 20,\n"
                   "    gridLengthFactor: 2,\n"
                   "    maxTime: 0.003,\n"
                   "    checkCoordX: 0.8,\n"
                   "    checkCoordY: 0.8,\n"
                   "    checkCoordZ: 0.8,\n"
                   "    sceneInfo: [\n"
                   "    \t{\n"
                   '    \t    name: "sphere",\n'
                   '    \t    type: "Audio"\n'
                   "    \t},\n"
                   "    \t{\n"
                   '    \t    name: "cube",\n'
                   '    \t    type: "Modal"\n'
                   "    \t}\n"
                   "    ]\n"
                   "}\n" % (scene, out))
    r = subprocess.run([DEMO, str(cfg)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr + r.stdout
    vals = np.array([float(x) for x in (out / "result.txt").read_text().split()])
    rate = int(vals[0])
    assert rate > 0 and abs(vals[0] - rate) == 0
    samples = vals[1:]
    # silent lead-in: the modal IIR is stepped at the step rate up to the first contact (2 ms);
    # that many samples lead the output (float arithmetic as in the host)
    dt = np.float32(1.0) / np.float32(rate)
    t = np.float32(0)
    while t + dt < np.float32(0.002):
        t = np.float32(t + dt)
    mute = int(np.float32(t * np.float32(rate)))
    frame_num = int(np.float32(0.003) / dt)
    assert 0.002 * rate - 3 <= mute <= 0.002 * rate + 1
    assert abs(len(samples) - (mute + frame_num + 1)) <= 1
    assert np.all(samples[:mute] == 0)
    # then maxTime of steps, finite and sounding
    assert np.all(np.isfinite(samples)) and np.abs(samples[mute:]).max() > 0
