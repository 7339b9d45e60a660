"""Host-side pieces that need no GPU: the spin-file format, the C driver's
argument handling, and that the C programs fail loudly without a device."""
from __future__ import annotations

import subprocess

import numpy as np
import pytest

import asd_b200 as asd
from conftest import PKG, ROOT

HOST = PKG / "host" / "llg_sqt"


def test_spin_file_round_trip(tmp_path):
    s = asd.random_spins(6, 3, seed=2)
    p = tmp_path / "a.spins"
    asd.save_spins(p, s, step=17, spin_len=1.0)
    got, step, slen = asd.load_spins(p)
    assert np.array_equal(got, s) and step == 17 and slen == 1.0
    assert p.stat().st_size == 64 + s.size * 8


def test_spin_file_errors(tmp_path):
    bad = tmp_path / "bad.spins"
    bad.write_bytes(b"NOTSPINS" + bytes(56))
    with pytest.raises(asd.AsdError):
        asd.load_spins(bad)
    s = asd.random_spins(4, 2, seed=1)
    p = tmp_path / "t.spins"
    asd.save_spins(p, s)
    p.write_bytes(p.read_bytes()[:-8])  # truncated
    with pytest.raises(asd.AsdError):
        asd.load_spins(p)
    with pytest.raises(asd.AsdError):
        asd.load_spins(tmp_path / "missing.spins")


@pytest.fixture(scope="module")
def host_bin():
    subprocess.run(["make", "-C", str(PKG), "host/llg_sqt"], check=True, capture_output=True)
    return HOST


def test_host_rejects_bad_arguments(host_bin):
    r = subprocess.run([str(host_bin), "-q", "fp16"], capture_output=True, text=True)
    assert r.returncode == 2 and "usage" in r.stderr
    r = subprocess.run([str(host_bin), "-H", "1,2"], capture_output=True, text=True)
    assert r.returncode == 2


def test_host_has_no_cpu_fallback(host_bin):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    r = subprocess.run([str(host_bin), "-n", "8", "-f", "2", "-m", "2"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and "CUDA" in r.stderr
    for mode in ("fp64", "tf32x3", "bf16x3", "fp16x3"):  # every mode parses; none runs on the CPU
        r = subprocess.run([str(host_bin), "-n", "8", "-f", "2", "-m", "2", "-q", mode],
                           capture_output=True, text=True)
        assert r.returncode == 1 and "CUDA" in r.stderr, mode


def test_dropin_program_links_against_the_library(tmp_path):
    exe = tmp_path / "dropin_host"
    subprocess.run(["gcc", "-O2", "-o", str(exe), str(ROOT / "tests" / "dropin_host.c"),
                    f"-I{ROOT / 'include'}", f"-L{PKG / 'lib'}", "-lasd_b200",
                    f"-Wl,-rpath,{PKG / 'lib'}", "-lm"], check=True)
    out = subprocess.run(["nm", "-D", "--defined-only", str(exe)], capture_output=True,
                         text=True).stdout
    # the program exports the reference's globals for the library's weak references
    for g in ("N", "Nfile", "J1", "dt"):
        assert f" {g}\n" in out or out.endswith(f" {g}")
