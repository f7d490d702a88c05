"""The drop-in drivers (sgtpsv / sgtsh): reference stdin and file formats.

CPU: the inputs parse and, without a device, the run stops with an error
after reading them.  GPU: a small P-SV run writes one catalogue file per
(receiver, frequency) with the reference's names and record size, holding
the complex64 cast of the golden (oracle) result."""
import os
import subprocess

import numpy as np
import pytest

import dsmsgt
from dsmsgt import synth
from conftest import REPO, rel_l2

BIN = os.path.join(REPO, "dsm-kernel_b200", "bin")


def write_inputs(tmp, imax, freqs_case=True):
    (tmp / "DSM.config").write_text(synth.dsm_config())
    (tmp / "model.psv.model").write_text(synth.psv_earth_model(0))
    par = synth.param_file(tlen=1638.4, rmin=1000.0, rmax=6300.0, rdelta=500.0, r0=6071.0,
                           thmin=0.0, thmax=180.0, thdelta=15.0, imin=0, imax=imax,
                           modelname="synth", outdir=str(tmp / "out"),
                           conf=str(tmp / "DSM.config"), model=str(tmp / "model.psv.model"))
    (tmp / "param").write_text(par)
    return par


def test_driver_reads_inputs_without_device(built, tmp_path):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    write_inputs(tmp_path, 4)
    with open(tmp_path / "param") as f:
        p = subprocess.run([os.path.join(BIN, "sgtpsv")], stdin=f, capture_output=True, text=True)
    assert p.returncode == 1
    assert "context" in p.stderr and "device" in p.stderr


def i7(v):
    return f"{int(v):7d}"


@pytest.mark.gpu
def test_driver_writes_reference_catalogue(built, tmp_path):
    imax = 64  # the grid depends on imax: same as the golden case
    write_inputs(tmp_path, imax)
    with open(tmp_path / "param") as f:
        p = subprocess.run([os.path.join(BIN, "sgtpsv")], stdin=f, capture_output=True, text=True,
                           timeout=600)
    assert p.returncode == 0, p.stderr
    g = np.load(os.path.join(REPO, "tests", "golden", "psv_small_seed0.npz"))
    s = dsmsgt.Setup(__import__("cases").psv_small(), "psv")
    r = np.ctypeslib.as_array(s.s.r, shape=(s.r_n,))
    out = tmp_path / "out"
    tsgt_files = os.listdir(out / "TSGT")
    assert len(tsgt_files) == s.r_n * imax
    for k, i in enumerate(g["freqs"]):
        if i > imax:
            continue
        got = np.zeros((s.r_n, s.theta_n, 20), np.complex64)
        for ir in range(s.r_n):
            name = (i7(6071.0 * 1e3) + "." + i7(r[ir] * 1e3) + "." + i7(i) + ".TSGT_PSV")
            name = name[:29].replace(" ", "0") + name[29:]
            raw = np.fromfile(out / "TSGT" / f"synth.{name}", dtype=np.complex64)
            assert raw.size == 20 * s.theta_n  # recl = 2 num 4 theta bytes
            got[ir] = raw.reshape(s.theta_n, 20)
        ref = np.transpose(g["tsgt"][k], (1, 0, 2))  # [itheta][ir][comp] -> [ir][itheta][comp]
        assert rel_l2(got.astype(np.complex128), ref) <= 1e-6
        syn = (i7(6071.0 * 1e3) + "." + i7(i) + ".SYNN_PSV")
        syn = syn[:21].replace(" ", "0") + syn[21:]
        assert os.path.getsize(out / "RSGT" / f"synth.{syn}") == 8 * 10 * s.theta_n
    logs = os.listdir(out / "log")
    assert any(n.startswith("calLog.synth.") for n in logs)
    lst = [n for n in logs if n.startswith("list.synth.")]
    assert len(lst) == 1
    lines = [ln.split() for ln in open(out / "log" / lst[0]).read().splitlines() if ln.strip()]
    assert [int(ln[0]) for ln in lines] == sorted(int(ln[0]) for ln in lines)
    assert len(lines) == imax
