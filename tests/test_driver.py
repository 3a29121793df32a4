"""The C drop-in driver amber_gpu: reference inputs in, byte-compatible files out."""
import glob
import json
import os
import subprocess

import numpy as np
import pytest

import oracle
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
    absscale = [o["absscale"] for o in oracle.estimate(real, version=1, with_absscale=True)[1]] \
        if precision == "mixed" else None
    rd = formats.read_closed_rings(str(res))
    np.testing.assert_array_equal(rd[:, :3], z["rdata"][:, :3])
    n = real.nclen
    for i, (r1, r2, r3, _) in enumerate(z["rdata"]):
        f = os.path.join(res, formats.bsout_name(1, int(r1), int(r2), int(r3), 1))
        assert os.path.getsize(f) == 16 + n * n * 8  # the reference's v1 layout
        ntri, num, bl, nd = formats.read_bsout_v1(f, n)
        np.testing.assert_allclose([ntri, num], [z["ntri"][i], z["num"][i]], rtol=1e-10)
        np.testing.assert_array_equal(nd, z["numdnu"][i])
        if precision == "fp64":
            # float file values: within the reference float build's own rounding of the FP64 result
            scale = np.abs(z["bldnu64"][i]).max()
            assert np.abs(bl - z["bldnu64"][i]).max() <= 1e-6 * scale
        else:
            # the mixed path's bound, 1e-6 of Σ|products| per lag cell, plus the file's float rounding
            e = np.abs(bl - z["bldnu64"][i]) / (absscale[i] + 1e-300)
            assert e.max() <= 1e-6 + 6e-8 * (np.abs(z["bldnu64"][i]) / (absscale[i] + 1e-300)).max(), e.max()


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


@pytest.mark.parametrize("version", [1, 2])
def test_driver_sharded_ranks_write_the_single_process_files(tmp_path, version):
    """Under RANK / WORLD_SIZE each process writes only its share of the triangles (the library's
    shard plan), and the union of the ranks' files is byte for byte the single-process output.
    The two ranks run one after the other on the same GPU (nothing waits on the other)."""
    from amber_b200 import build
    build.build()
    z = np.load(os.path.join(GOLDEN, "est_flagged48.npz"))
    real = _real_from(z)
    single, _ = _run(real, tmp_path, version, "mixed")
    exe = os.path.join(os.path.dirname(build.LIB), "amber_gpu")
    shared = tmp_path / "sharded"
    counts = []
    for rank in range(2):
        env = dict(os.environ, RANK=str(rank), WORLD_SIZE="2", LOCAL_RANK="0")
        p = subprocess.run([exe, "1", f"v{version}", str(real.nc10), str(tmp_path / "rings.txt"), "0", "-1",
                            str(shared), str(tmp_path / "input_params_ess"), "mixed"],
                           capture_output=True, text=True, cwd=tmp_path, env=env)
        assert p.returncode == 0, p.stderr
        st = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("AMBER_GPU_JSON ")][-1][15:])
        assert (st["rank"], st["world"]) == (rank, 2)
        counts.append(st["triangles"])
    assert sum(counts) == len(z["rdata"]) and min(counts) > 0
    names = sorted(os.listdir(single))
    assert names == sorted(os.listdir(shared))
    for n in names:
        with open(os.path.join(single, n), "rb") as a, open(os.path.join(shared, n), "rb") as b:
            assert a.read() == b.read(), n


def _run_vcg(tmp, z, collapse, fwhm=1480.73):
    from amber_b200 import build
    build.build()
    vis = tmp / "vis.bin"
    formats.write_vis(vis, z["randpar"], z["data"], np.float32(z["nu0"]), 40.0e3, 1.0)
    params = tmp / "inputparameters"
    params.write_text(f"{z['data'].shape[1]}\t{float(z['umax'])!r}\t{fwhm!r}\t1.\n")
    gv, smp = tmp / "GV_gpu", tmp / "sampling_gpu"
    exe = build.VCG_DRIVER
    p = subprocess.run([exe, str(vis), str(params), str(gv), str(int(z["flag_key"])), str(int(collapse)), "1",
                        str(smp)], capture_output=True, text=True, cwd=tmp)
    assert p.returncode == 0, p.stderr
    stats = json.loads([ln for ln in p.stdout.splitlines() if ln.startswith("VCG_GPU_JSON ")][-1][13:])
    return gv, smp, stats


@pytest.mark.parametrize("case,collapse", [("grid_coll_flag1", True), ("grid_flag0", False)])
def test_vcg_driver_matches_reference_files(tmp_path, case, collapse):
    """vcg_gpu (the gridding stage's executable): same arguments, same GV and sampling files as the
    reference's 3_vcg run on the same records (bit-identical values; byte-identical files when the
    reference build is present)."""
    import oracle
    z = np.load(os.path.join(GOLDEN, case + ".npz"))
    fwhm = float(z["fwhm"]) if "fwhm" in z.files else 1480.73
    gv_path, smp_path, stats = _run_vcg(tmp_path, z, collapse, fwhm)
    nc_out = z["gv"].shape[2]
    assert stats["NN"] == int(z["nn"]) and stats["nc_out"] == nc_out and stats["dU"] == float(z["du"])
    assert os.path.getsize(gv_path) == 28 + z["gv"].size * 16
    gv, du, fk = formats.read_gv(gv_path)
    assert du == float(z["du"]) and fk == int(z["flag_key"])
    assert np.array_equal(gv.real, z["gv"].real) and np.array_equal(gv.imag, z["gv"].imag)
    assert np.array_equal(formats.read_sampling(smp_path, int(z["nn"]), nc_out), z["ntig"])
    if oracle.ref_available():
        ref = tmp_path / "ref"
        ref.mkdir()
        vis = tmp_path / "vis.bin"
        params = tmp_path / "inputparameters"
        p = subprocess.run([os.path.join(oracle.REF_DIR, "ref_vcg"), str(vis), str(params), str(ref / "GV"),
                            str(int(z["flag_key"])), str(int(collapse)), "1", str(ref / "sampling")],
                           capture_output=True, text=True, cwd=ref)
        assert p.returncode == 0, p.stdout[-500:]
        assert (ref / "GV").read_bytes() == gv_path.read_bytes()
        assert (ref / "sampling").read_bytes() == smp_path.read_bytes()
