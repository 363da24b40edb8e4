"""The C ABI library loads on a machine without a GPU and exports every symbol the header
declares; the checkers load too.  No compute call is made here."""
import ctypes
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "pppm_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(pppm_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_the_boundary():
    names = header_functions()
    for required in ("pppm_create", "pppm_destroy", "pppm_set_mesh", "pppm_update_mesh", "pppm_step",
                     "pppm_add_listener", "pppm_read_listeners", "pppm_save_state", "pppm_restore_state",
                     "pppm_reset_fields", "pppm_dump", "pppm_import_grid_cache", "pppm_import_face_cache",
                     "pppm_batch_create", "pppm_batch_run", "pppm_adjoint"):
        assert required in names


def test_library_exports_every_declared_symbol():
    import pppm_b200

    lib = ctypes.CDLL(pppm_b200.LIB_PATH)
    missing = [n for n in header_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings():
    import pppm_b200

    assert pppm_b200.lib.pppm_status_string(0) == b"ok"
    assert pppm_b200.lib.pppm_status_string(3) == b"capacity exceeded"


def test_create_rejects_bad_parameters_without_device_calls():
    import pppm_b200

    for kw in (dict(res=4, dl=0.01, dt=1e-5), dict(res=32, dl=-1.0, dt=1e-5), dict(res=32, dl=0.01, dt=1e-5, pml_width=40)):
        try:
            pppm_b200.Solver(**kw)
        except pppm_b200.PPPMError as e:
            assert e.status == pppm_b200.ERR_ARG
        else:
            raise AssertionError("accepted %r" % kw)


def test_oracle_library_loads():
    from oracle.oracle import oracle_lib, oracle_threads

    assert oracle_lib() is not None
    assert oracle_threads() >= 1


def test_package_import_maps_no_native_code():
    """Importing the package (for its scene generators, as the benchmark's reference arm does)
    loads no native library; the first call through the library maps it."""
    import subprocess
    import sys

    code = ("import sys; sys.path.insert(0, %r); import pppm_b200; from pppm_b200 import scenes; "
            "maps = open('/proc/self/maps').read(); assert 'libpppm_b200' not in maps, 'mapped at import'; "
            "assert not pppm_b200.loaded(); pppm_b200.lib.pppm_status_string(0); "
            "assert 'libpppm_b200' in open('/proc/self/maps').read(); print('ok')"
            % os.path.join(ROOT, "pppm-tdbem_b200", "python"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stderr
