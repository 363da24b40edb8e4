"""The scene host `pppm_demo CONFIG` against the reference's own scene layer on the B200.

oracle/_ref/ref_demo runs the same config through the reference's SimpleJsonReader,
ObjectCollection (Audio, Manual and Modal objects: Object.h/.cu, ObjectCollection.cu,
RigidBody.cu) and PPPMSolver in the order of the demo driver (experiments/demo/main.cu:38-275),
with the identity mesh repair in place of its pymesh docker call (the test meshes are clean).
Three scenes, each in the reference's file layout:

  * a moving Audio sphere (mesh.obj, motion.txt frames with a rotation quaternion, accs.txt at
    44.1 kHz) beside a Manual plate (mesh.obj only);
  * the Audio sphere with selected_vertices.txt (only the faces that cover those vertices carry
    the acceleration, Object.cu:38-70) and the chunked cross-fade restart (chunkSize 40,
    backStepSize 12: main.cu:212-263);
  * a Modal cube (tet mesh, eigenmodes, contact impulses: the silent lead-in to the first contact,
    the damped modal IIR) beside the Audio sphere.

result.txt must have the reference's layout (line 0 the frame rate, one "%e" sample per step, the
same length and silent lead-in) and its samples must agree: within 1e-5 relative L2 over the
first 50 sounding steps where both sides read the same accelerations (Audio: accs.txt held per
44.1 kHz sample), 5e-5 with a Modal object (each side evaluates the modal recursion in its own
arithmetic: the reference's float kernels on the device, the host's loop here), and over the
whole run within twice the spread of two reference runs (its float atomics sum in a different
order each run), at least 1e-4.  Figures go to
$PPPM_METRICS_DIR/demo_parity_metrics.json when that variable is set.
"""
import json
import math
import os
import subprocess

import numpy as np
import pytest

from helpers import rel_l2
from pppm_b200 import scenes

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEMO = os.path.join(ROOT, "pppm-tdbem_b200", "bin", "pppm_demo")
REF_DEMO = os.path.join(ROOT, "oracle", "_ref", "ref_demo")
METRICS = {}


@pytest.fixture(scope="module", autouse=True)
def write_metrics():
    yield
    d = os.environ.get("PPPM_METRICS_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "demo_parity_metrics.json"), "w") as f:
            json.dump(METRICS, f, indent=1, default=float)


def _write_obj(path, v, f):
    with open(path, "w") as fo:
        for p in v:
            fo.write("v %.7f %.7f %.7f\n" % tuple(p))
        for t in f:
            fo.write("f %d %d %d\n" % tuple(np.asarray(t) + 1))


def _audio(d, selected=None):
    os.makedirs(d)
    v, f = scenes.icosphere(2)
    _write_obj(os.path.join(d, "mesh.obj"), v * 0.05, f)
    with open(os.path.join(d, "motion.txt"), "w") as fo:
        for k in range(6):  # a frame every 0.4 ms: translation along x and a rotation about z
            t = 0.0004 * k
            a = 0.3 * k
            fo.write("%.6f %.6f 0 0 0 0 %.6f %.6f\n" % (t, 0.004 * k, math.sin(a / 2), math.cos(a / 2)))
    acc = np.sin(2 * math.pi * 1500.0 * np.arange(200) / 44100.0)
    np.savetxt(os.path.join(d, "accs.txt"), acc, fmt="%.7f")
    if selected is not None:
        with open(os.path.join(d, "selected_vertices.txt"), "w") as fo:
            fo.write(" ".join(str(int(i)) for i in selected))


def _plate(d):
    os.makedirs(d)
    v, f = scenes.plate(4, 4, 0.16, 0.16, -0.09)
    _write_obj(os.path.join(d, "mesh.obj"), v, f)


def _modal(d, rng):
    os.makedirs(d)
    v = np.array([[x, y, z] for x in (0, 1) for y in (0, 1) for z in (0, 1)], float) * 0.05
    tets = np.array([[0, 1, 2, 4], [3, 1, 2, 7], [5, 1, 4, 7], [6, 2, 4, 7], [1, 2, 4, 7]])
    np.savetxt(os.path.join(d, "vertices.txt"), v, fmt="%.7g")
    np.savetxt(os.path.join(d, "tets.txt"), tets.astype(float), fmt="%.1f")
    lam = (2 * math.pi * np.array([800.0, 2100.0, 5200.0])) ** 2
    np.savetxt(os.path.join(d, "eigenvalues.txt"), lam, fmt="%.9g")
    np.savetxt(os.path.join(d, "eigenvectors.txt"), rng.standard_normal((24, 3)), fmt="%.7g")
    # frames past the end of the run: the reference's RigidBody indexes its frame times without a
    # bound (RigidBody.cu:313 in get_bbox, :333 in audio_step), so its motion list has to outlast
    # the run and hold a frame at or after the first contact
    with open(os.path.join(d, "motion.txt"), "w") as fo:
        for k in range(11):
            fo.write("%.4f 0.1 -0.025 -0.025 0 0 0 1\n" % (0.0005 * k))
    with open(os.path.join(d, "contact.txt"), "w") as fo:
        fo.write("0.001 7 0 0 1 3.0\n0.0014 0 1 0 0 1.0\n")


def _config(path, scene, out, objects, chunk=1000000, back=0, max_time=0.002):
    lines = ["{", '    inputDir: "%s",' % scene, '    outputDir: "%s",' % out, "    res: 24,",
             "    gridLengthFactor: 2,", "    reflectCoeff: 0.83,", "    maxTime: %g," % max_time,
             "    startTime: 0,", "    chunkSize: %d," % chunk, "    backStepSize: %d," % back,
             "    checkCoordX: 0.8,", "    checkCoordY: 0.7,", "    checkCoordZ: 0.75,", "    sceneInfo: ["]
    for i, (name, kind) in enumerate(objects):
        lines += ["    \t{", '    \t    name: "%s",' % name, '    \t    type: "%s"' % kind,
                  "    \t}," if i + 1 < len(objects) else "    \t}"]
    lines += ["    ]", "}"]
    with open(path, "w") as fo:
        fo.write("\n".join(lines) + "\n")


def _run(exe, cfg, out):
    r = subprocess.run([exe, str(cfg)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, (exe, r.stderr[-2000:], r.stdout[-2000:])
    text = (out / "result.txt").read_text()
    return text, np.array([float(x) for x in text.split()])


SCENES = {
    "audio_manual": dict(objects=[("sphere", "Audio"), ("plate", "Manual")]),
    "selected_crossfade": dict(objects=[("sphere", "Audio")], chunk=40, back=12, selected=True),
    "modal_audio": dict(objects=[("cube", "Modal"), ("sphere", "Audio")], early=5e-5),
}


@pytest.mark.parametrize("name", sorted(SCENES))
def test_demo_matches_reference_scene_layer(gpu, tmp_path, name):
    if not (os.path.exists(DEMO) and os.path.exists(REF_DEMO)):
        pytest.skip("scene host or reference demo not built")
    spec = SCENES[name]
    scene = tmp_path / "scene"
    rng = np.random.default_rng(5)
    for obj, kind in spec["objects"]:
        if kind == "Audio":
            sel = None
            if spec.get("selected"):
                sel = np.random.default_rng(9).choice(162, 40, replace=False)
            _audio(str(scene / obj), sel)
        elif kind == "Manual":
            _plate(str(scene / obj))
        else:
            _modal(str(scene / obj), rng)
    runs = {}
    for who, exe in (("ours", DEMO), ("ref", REF_DEMO), ("ref2", REF_DEMO)):
        out = tmp_path / ("out_" + who)
        cfg = tmp_path / ("%s.cfg" % who)
        _config(cfg, scene, out, spec["objects"], spec.get("chunk", 1000000), spec.get("back", 0))
        runs[who] = _run(exe, cfg, out)
    (t_ours, ours), (t_ref, ref), (_, ref2) = runs["ours"], runs["ref"], runs["ref2"]
    # layout: same line count, frame rate on line 0, no trailing newline, "%e" samples
    assert len(t_ours.split("\n")) == len(t_ref.split("\n"))
    assert not t_ours.endswith("\n") and not t_ref.endswith("\n")
    assert t_ours.split("\n")[0] == t_ref.split("\n")[0]
    assert len(ours) == len(ref)
    s_ours, s_ref, s_ref2 = ours[1:], ref[1:], ref2[1:]
    lead = int(np.argmax(s_ref != 0)) if np.any(s_ref != 0) else len(s_ref)
    lead_ours = int(np.argmax(s_ours != 0)) if np.any(s_ours != 0) else len(s_ours)
    spread = rel_l2(s_ref2, s_ref)
    early = slice(lead, lead + 50)
    METRICS[name] = {"samples": int(len(s_ref)), "frame_rate": float(ref[0]), "silent_lead_in": lead,
                     "rel_l2_first50": rel_l2(s_ours[early], s_ref[early]), "rel_l2_all": rel_l2(s_ours, s_ref),
                     "reference_spread": spread}
    assert lead_ours == lead
    assert np.all(np.isfinite(s_ours)) and np.abs(s_ours).max() > 0
    assert rel_l2(s_ours[early], s_ref[early]) < spec.get("early", 1e-5)
    assert rel_l2(s_ours, s_ref) < max(2 * spread, 1e-4)
