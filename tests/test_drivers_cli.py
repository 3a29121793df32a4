"""The drop-in executables' argument and input handling, before any GPU work (runs on CPU)."""
import os
import subprocess

import numpy as np
import pytest

import amber_b200
from amber_b200 import build, formats, synth


@pytest.fixture(scope="module")
def exes():
    build.build()
    return build


def _run(args, cwd):
    return subprocess.run(args, capture_output=True, text=True, cwd=cwd)


def test_vcg_usage_and_bad_keys(exes, tmp_path):
    p = _run([exes.VCG_DRIVER], tmp_path)
    assert p.returncode == 1 and "Usage" in p.stdout
    p = _run([exes.VCG_DRIVER, "vis", "params", "GV", "2", "0", "1", "samp"], tmp_path)
    assert p.returncode == 1 and "0 or 1" in p.stderr


def test_vcg_rejects_a_file_that_is_not_visibilities(exes, tmp_path):
    (tmp_path / "params").write_text("4\t20.0\t1480.73\t1.\n")
    (tmp_path / "vis").write_bytes(b"NOTAVIS!" + bytes(64))
    p = _run([exes.VCG_DRIVER, "vis", "params", "GV", "1", "0", "1", "samp"], tmp_path)
    assert p.returncode == 1 and "not a visibility file" in p.stderr


@pytest.mark.parametrize("g,pcount,nstokes,nchan", [(-1, 5, 2, 8), (1 << 40, 5, 2, 8), (10, 1 << 30, 2, 8),
                                                     (10, 5, 1 << 20, 8), (10, 5, 2, 1 << 40)])
def test_vcg_rejects_a_visibility_header_out_of_range(exes, tmp_path, g, pcount, nstokes, nchan):
    """Record, parameter, Stokes and channel counts past what any file holds are refused as "not a
    visibility file" before any buffer is sized from them."""
    (tmp_path / "params").write_text("4\t20.0\t1480.73\t1.\n")
    with open(tmp_path / "vis", "wb") as f:
        f.write(formats.VIS_HEADER.pack(formats.VIS_MAGIC, g, pcount, nstokes, nchan, 1.5e8, 4e4, 1.0, 0.0))
        f.write(bytes(64))
    p = _run([exes.VCG_DRIVER, "vis", "params", "GV", "1", "0", "1", "samp"], tmp_path)
    assert p.returncode == 1 and "not a visibility file" in p.stderr, p.stderr


def test_vcg_rejects_more_channels_than_the_file_holds(exes, tmp_path):
    randpar, data = synth.make_visibilities(16, 1.0254384902642049, 3, 20, 5, umax=8.0)
    formats.write_vis(tmp_path / "vis", randpar, data, np.float32(synth.NU0), 40.0e3, 1.0)
    (tmp_path / "params").write_text("5\t8.0\t1480.73\t1.\n")
    p = _run([exes.VCG_DRIVER, "vis", "params", "GV", "1", "0", "1", "samp"], tmp_path)
    assert p.returncode == 1 and "holds 3" in p.stderr


def test_amber_gpu_runs_on_the_reference_defaults(exes, tmp_path):
    """`amber_gpu <Rlzn>` alone, as `amber <Rlzn>` is run: the version, nc10 and rings default to the
    reference's (v1, nc10 = 383, the annular_rings edges), so it goes straight to its inputs."""
    p = _run([exes.DRIVER], tmp_path)
    assert p.returncode == 1 and "Usage" in p.stdout
    p = _run([exes.DRIVER, "1"], tmp_path)
    assert p.returncode != 0 and "input_params_ess" in p.stderr


def test_amber_gpu_default_rings_are_the_reference_annular_rings(exes):
    """The driver's default ring edges equal those the reference's own annular_rings() sets
    (4_fbe/amber_funcs.c:2022-2062 compiled unchanged into oracle/_ref/ref_rings), for the 22 bins
    of amber.c:44-45, digit for digit."""
    import oracle
    ref = os.path.join(oracle.REF_DIR, "ref_rings")
    if not os.path.exists(ref):
        pytest.skip("reference build oracle/_ref missing (make -C oracle ref)")
    ours = subprocess.run([exes.DRIVER, "--default-rings"], capture_output=True, text=True, check=True).stdout
    theirs = subprocess.run([ref], capture_output=True, text=True, check=True).stdout
    assert ours == theirs
    lines = ours.split("\n")
    assert lines[0] == "22" and lines[1] == "1 5" and lines[22] == "235 270"


def test_maps_usage_and_missing_inputs(exes, tmp_path):
    p = _run([exes.MAPS_DRIVER], tmp_path)
    assert p.returncode == 1 and "Usage" in p.stdout
    p = _run([exes.MAPS_DRIVER, "1", "GV_data_1"], tmp_path)
    assert p.returncode != 0 and "input_params" in p.stderr
    (tmp_path / "input_params").write_text(f"32\t0.5\t154.255e6\t40e3\t1\t8\t{tmp_path / 'nowhere'}\n")
    p = _run([exes.MAPS_DRIVER, "1", "GV_data_1"], tmp_path)
    assert p.returncode != 0 and "GV_data" in p.stderr


def _bad_grid(path, nn, nc, du):
    """A GV_data file whose 28-byte header (formats.GV_HEADER) holds the given values, then a little
    data: the drivers must refuse it before sizing any buffer from it."""
    with open(path, "wb") as f:
        f.write(formats.GV_HEADER.pack(nn, nc, du, 0))
        f.write(bytes(256))


@pytest.mark.parametrize("nn,nc,du", [(-4, 3, 0.5), (15, 3, 0.5), (16, 0, 0.5), (16, 3, 0.0),
                                      (1 << 40, 1 << 40, 0.5)])
def test_drivers_refuse_a_grid_header_that_is_not_a_grid(exes, tmp_path, nn, nc, du):
    """A negative, odd or absurd side, no channels or a non-positive cell size: both executables
    stop with "bad header" and a failure status (the sizes would otherwise wrap malloc and fread)."""
    data = tmp_path / "data"
    data.mkdir()
    _bad_grid(data / "GV_data_1", nn, nc, du)
    formats.write_input_params_ess(tmp_path / "input_params_ess", 154.255, 0.04, 1.0, str(data))
    p = _run([exes.DRIVER, "1"], tmp_path)
    assert p.returncode != 0 and "bad header" in p.stderr, p.stderr
    (tmp_path / "input_params").write_text(f"32\t0.5\t154.255e6\t40e3\t1\t8\t{data}\n")
    p = _run([exes.MAPS_DRIVER, "1", "GV_data_1"], tmp_path)
    assert p.returncode != 0 and "bad header" in p.stderr, p.stderr


def test_cylbs_parameter_checks():
    with pytest.raises(ValueError):
        amber_b200.cylbs_params(denominator="both")
    with pytest.raises(TypeError):
        amber_b200.cylbs_params(n_kut=3)
    p = amber_b200.cylbs_params(window=True, denominator="mask", n_cut=3)
    assert (p.n_cut, p.window, p.denominator) == (3, 1, 1)
    assert p.mabs_norm == amber_b200.reference_cylbs_constants()["mabs_norm"]


def test_grid_vis_rejects_bad_record_shapes():
    """The Python wrapper checks the record arrays before any library call (no GPU needed)."""
    est = amber_b200.Estimator.__new__(amber_b200.Estimator)  # no context: the checks come first
    randpar = np.zeros((5, 3), dtype=np.float32)
    for bad in (np.zeros((5, 3, 2), np.float32),        # not [G, nchan, nstokes, 3]
                np.zeros((5, 2, 1, 3), np.float32),     # fewer channels than nc
                np.zeros((4, 3, 1, 3), np.float32),     # record count differs from randpar
                np.zeros((5, 3, 1, 2), np.float32)):    # not (re, im, wt)
        with pytest.raises(ValueError):
            est.grid_vis(16, 3, 0.5, 4.0, 1.5e8, 1, randpar, bad)
