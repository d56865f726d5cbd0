"""CPU checks of the drop-in boundary: libbeatbox.so loads without a GPU, exports every entry
point include/beatbox.h declares, and the ctypes struct layouts match the C header."""
import ctypes
import os
import re
import subprocess

import pytest

import beatbox

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "beatbox.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(bb_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("bb_world_create", "bb_world_destroy", "bb_add_box_shape", "bb_add_sphere_shape", "bb_add_bodies",
                 "bb_set_material", "bb_set_solver_params", "bb_step", "bb_read_state", "bb_read_stats"):
        assert must in names


def test_library_loads_and_exports_every_declared_symbol():
    lib = beatbox.load_library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert b"sm_100a" in lib.bb_version()
    # every symbol the Python wrapper binds exists in the header too
    assert set(beatbox._SIG) <= set(declared_functions())


def test_default_params_are_the_reference_constants():
    p = beatbox.default_params()
    assert p.solver == beatbox.SOLVER_AVBD and p.iterations == 5 and p.gc_rounds == 32
    assert p.flags == beatbox.SIM_DEFAULT_FLAGS and p.quirks == beatbox.QUIRKS_REFERENCE
    assert abs(p.gravity + 9.81) < 1e-6 and abs(p.penetration_cap + 0.25) < 1e-7
    assert p.avbd_iterations == 10 and p.avbd_beta == 100000.0 and abs(p.avbd_gamma - 0.99) < 1e-7
    assert p.avbd_shock_layers == 12 and p.avbd_post_stab_sweeps == 4 and p.avbd_color_rounds == 16
    assert list(p.world_min) == [-64.0] * 3 and list(p.world_extent) == [128.0] * 3


def _c_sizeof(struct: str) -> int:
    code = f'#include "{HEADER}"\n#include <stdio.h>\nint main(){{printf("%zu", sizeof({struct}));return 0;}}\n'
    exe = os.path.join("/tmp", f"bb_sizeof_{struct}")
    src = exe + ".c"
    open(src, "w").write(code)
    subprocess.check_call(["gcc", "-o", exe, src])
    return int(subprocess.check_output([exe]).decode())


@pytest.mark.parametrize("struct,cls", [("bb_solver_params", beatbox.SolverParams), ("bb_world_desc", beatbox.WorldDesc),
                                        ("bb_body_desc", beatbox.BodyDesc), ("bb_step_stats", beatbox.StepStats)])
def test_ctypes_layout_matches_header(struct, cls):
    assert _c_sizeof(struct) == ctypes.sizeof(cls)


def test_oracle_stats_struct_matches_header():
    import pyoracle

    assert _c_sizeof("bb_step_stats") == ctypes.sizeof(pyoracle.StepStats)


def test_record_dtypes_match_header():
    assert _c_sizeof("bb_manifold_info") == beatbox.MANIFOLD_DTYPE.itemsize
    assert _c_sizeof("bb_contact_info") == beatbox.CONTACT_DTYPE.itemsize


def test_world_creation_fails_loudly_without_gpu():
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("a GPU is present")
    with pytest.raises(beatbox.BeatboxError):
        beatbox.World(16)
