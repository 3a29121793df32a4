"""The C drop-in driver amber_gpu: reference inputs in, byte-compatible files out."""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

from amber_b200 import formats, synth

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _real_from(z):
    return synth.Realisation(nn=z["gv"].shape[0], nc=z["gv"].shape[2], du=float(z["du"]), flag_key=int(z["flag_key"]),
                             gv=z["gv"], counts=z["counts"], uf_chans=z["uf_chans"], ulow=z["ulow"],
                             uhigh=z["uhigh"], nc10=int(z["nc10"]), seed=0)


def _run(real, tmp, version, precision):
    from amber_b200 import build
    build.build()
    data = tmp / "data"
    real.write(str(data), 1)
    formats.write_input_params_ess(tmp / "input_params_ess", 154.255e6, 40.0e3, 1.0, str(data))
    formats.write_rings_file(tmp / "rings.txt", real.ulow, real.uhigh)
    res = tmp / f"res_{version}_{precision}"
    exe = os.path.join(os.path.dirname(build.LIB), "amber_gpu")
    p = subprocess.run([exe, "1", f"v{version}", str(real.nc10), str(tmp / "rings.txt"), "0", "-1", str(res),
                        str(tmp / "input_params_ess"), precision], capture_output=True, text=True, cwd=tmp)
    assert p.returncode == 0, p.stderr
    stats = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("AMBER_GPU_JSON ")][-1][15:])
    return res, stats


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_driver_v1_matches_reference_files(tmp_path, precision):
    z = np.load(os.path.join(GOLDEN, "est_flagged48.npz"))
    real = _real_from(z)
    res, stats = _run(real, tmp_path, 1, precision)
    assert stats["triangles"] == len(z["rdata"])
    rd = formats.read_closed_rings(str(res))
    np.testing.assert_array_equal(rd[:, :3], z["rdata"][:, :3])
    n = real.nclen
    for i, (r1, r2, r3, _) in enumerate(z["rdata"]):
        f = os.path.join(res, formats.bsout_name(1, int(r1), int(r2), int(r3), 1))
        assert os.path.getsize(f) == 16 + n * n * 8  # the reference's v1 layout
        ntri, num, bl, nd = formats.read_bsout_v1(f, n)
        np.testing.assert_allclose([ntri, num], [z["ntri"][i], z["num"][i]], rtol=1e-10)
        np.testing.assert_array_equal(nd, z["numdnu"][i])
        # float file values: within the reference float build's own rounding of the FP64 result
        scale = np.abs(z["bldnu64"][i]).max()
        assert np.abs(bl - z["bldnu64"][i]).max() <= 1e-6 * scale


def test_driver_v2_files(tmp_path):
    z = np.load(os.path.join(GOLDEN, "est_unflagged32.npz"))
    real = _real_from(z)
    res, _ = _run(real, tmp_path, 2, "mixed")
    n = real.nclen
    files = sorted(glob.glob(os.path.join(res, "bsout_final2_*")))
    assert len(files) == len(z["rdata"])
    for i, (r1, r2, r3, _) in enumerate(z["rdata"]):
        f = os.path.join(res, formats.bsout_name(2, int(r1), int(r2), int(r3), 1))
        assert os.path.getsize(f) == 8 + n * n * 8
        inv, bl, nt = formats.read_bsout_v2(f, n)
        assert inv == z["inv_ng"][i]
        assert np.abs(nt - z["numtri_v2"][i]).max() <= 1e-6 * np.abs(z["numtri_v2"][i]).max()
