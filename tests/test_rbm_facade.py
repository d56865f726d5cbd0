"""The C++ drop-in include/beatbox_rbm.hpp (the reference's RigidBodyManager surface,
src/rigid_body_manager.hpp:14-70), compiled with g++ and linked against libbeatbox.so: without
a GPU create() fails cleanly; on a GPU the facade's simulate() steps equal the C ABI's bit for
bit and read_back_sim_config() equals bb_read_stats."""
import os
import subprocess

import pytest

import beatbox

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "rbm_facade_check.cpp")


@pytest.fixture(scope="module")
def facade_exe(tmp_path_factory):
    beatbox.load_library()  # builds libbeatbox.so if missing
    out = str(tmp_path_factory.mktemp("rbm") / "rbm_facade_check")
    libdir = os.path.dirname(beatbox.LIB_PATH)
    subprocess.check_call(["g++", "-std=c++17", "-O1", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                           "-o", out, "-L", libdir, "-lbeatbox", f"-Wl,-rpath,{libdir}"])
    return out


def test_facade_compiles_and_create_fails_without_gpu(facade_exe):
    from conftest import gpu_available

    if gpu_available():
        pytest.skip("a GPU is present (the gpu test covers the facade)")
    r = subprocess.run([facade_exe, "nogpu"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and "ok nogpu" in r.stdout, r.stdout + r.stderr


@pytest.mark.gpu
def test_facade_simulate_equals_the_c_abi_bit_for_bit(facade_exe):
    r = subprocess.run([facade_exe, "gpu"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and "ok gpu" in r.stdout, r.stdout + r.stderr
