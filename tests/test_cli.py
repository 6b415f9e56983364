"""grid.out / dft.out command lines (flag syntax of src/grid/grid.cpp:107-190
and src/dft/dft.cpp:88-187): host-side behaviour, no device needed."""
import os
import subprocess

import pytest

BIN = os.path.join(os.path.dirname(__file__), "..", "radio-gridders_b200", "bin")


def run(name, *args, env=None):
    e = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    e.update(env or {})
    return subprocess.run([os.path.join(BIN, name), *args], capture_output=True, text=True, env=e, timeout=60)


@pytest.mark.parametrize("name", ["grid.out", "dft.out"])
def test_built(rg, name):
    assert os.access(os.path.join(BIN, name), os.X_OK)


def test_help_and_missing_inputs(rg):
    r = run("grid.out", "--help")
    assert r.returncode == 0 and "-subgrid" in r.stdout and "-wproj" in r.stdout
    r = run("grid.out", "-theta=0.1", "-lambda=5120")
    assert r.returncode == 0 and "No Visibility File Specified" in r.stdout
    r = run("grid.out", "-vis=x.h5", "-theta=0.1", "-lambda=5120")
    assert "No W-Kernel File Specified" in r.stdout
    # flags are case-insensitive with any number of leading dashes
    r = run("grid.out", "---VIS=x.h5", "-WKernel=k.h5", "-lambda=5120")
    assert "No theta given" in r.stdout
    r = run("grid.out", "-vis=x.h5", "-wkernel=k.h5", "-theta=0.1", "-lambda=5120", "-subgrid=128")
    assert "Missing W-Towers Parameters" in r.stdout
    r = run("dft.out", "-vis=x.h5")
    assert r.returncode == 0 and "No theta" in r.stdout


def test_no_device_is_an_error(rg):
    r = run("grid.out", "-vis=x.h5", "-wkernel=k.h5", "-theta=0.1", "-lambda=5120", "-wproj")
    assert r.returncode == 1 and "context" in r.stderr
