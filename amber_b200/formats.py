"""Binary file formats of the AMBER pipeline (readers and writers).

Every layout here is fixed by the reference, which the consumers
(``mabs_funcs.read_bsout_float`` / ``read_bsout_float_v2``) parse with no
header of dimensions:

* gridded visibilities ``GV_data_<R>`` — header ``{int64 NN; int64 nc;
  f64 Du; int32 flag_key}`` (28 bytes, unpadded), then for every cell
  ``ii < NN, jj < NN/2+1`` and channel ``nn < nc``: ``f64 re, f64 im``
  (3_vcg/tgefuncs.c:628-655; read back by 4_fbe/amber_funcs.c:1861-1900);
* sampling counts ``sampling`` — ``f64`` per cell and channel in the same
  order, no header (3_vcg/tgefuncs.c:728-748);
* ``uf_chans.txt`` — whitespace-separated unflagged channel indices
  (4_fbe/amber_funcs.c:2485-2508);
* ``input_params_ess`` — ``nu0 dnu chan0 data_path`` (amber_funcs.c:175-188);
* ``closed_rings`` — rcount × ``{f64 r1, r2, r3, Num}`` and ASCII ``rcount``
  (amber_funcs.c:406-483);
* v1 output ``bsout_final_ra{r1}_rb{r2}_rc{r3}_R{R}`` — ``{f64 Ntri, f64 Num,
  f32 bldnu[nclen²], i32 numdnu[nclen²]}`` (4_fbe/amber.c:287-304);
* v2 output ``bsout_final2_…`` — ``{f64 1/Ng1², f32 bldnu[nclen²],
  f32 numdnu[nclen²]}`` (4_fbe/amber_v2.c:295-309).

All native (little-endian) byte order.
"""
from __future__ import annotations

import os
import struct

import numpy as np

GV_HEADER = struct.Struct("<qqdi")  # 28 bytes, no padding


def write_gv(path, re_im: np.ndarray, du: float, flag_key: int) -> None:
    """Write a gridded-visibility file. ``re_im``: complex128 [NN, NN/2+1, nc]."""
    nn, h, nc = re_im.shape
    assert h == nn // 2 + 1
    with open(path, "wb") as f:
        f.write(GV_HEADER.pack(nn, nc, float(du), int(flag_key)))
        np.ascontiguousarray(re_im, dtype=np.complex128).tofile(f)


def read_gv(path):
    """Return (re_im complex128 [NN, H, nc], Du, flag_key)."""
    with open(path, "rb") as f:
        nn, nc, du, flag_key = GV_HEADER.unpack(f.read(GV_HEADER.size))
        h = nn // 2 + 1
        data = np.fromfile(f, dtype=np.complex128, count=nn * h * nc)
    if data.size != nn * h * nc:
        raise ValueError(f"{path}: truncated grid ({data.size} of {nn * h * nc} cells×channels)")
    return data.reshape(nn, h, nc), du, flag_key


def write_sampling(path, counts: np.ndarray) -> None:
    np.ascontiguousarray(counts, dtype=np.float64).tofile(path)


def read_sampling(path, nn: int, nc: int) -> np.ndarray:
    h = nn // 2 + 1
    data = np.fromfile(path, dtype=np.float64)
    if data.size < nn * h * nc:
        raise ValueError(f"{path}: truncated sampling file")
    return data[: nn * h * nc].reshape(nn, h, nc)


def write_uf_chans(path, chans) -> None:
    with open(path, "w") as f:
        f.write(" ".join(str(int(c)) for c in chans) + "\n")


def read_uf_chans(path, uf_nc: int) -> np.ndarray:
    """Read exactly ``uf_nc`` integers; a short file is an error (the reference
    returns -1 from get_uf_chans, amber_funcs.c:2497-2503)."""
    with open(path) as f:
        vals = [int(t) for t in f.read().split()]
    if len(vals) < uf_nc:
        raise ValueError(f"{path}: expected {uf_nc} integers, read {len(vals)}")
    return np.asarray(vals[:uf_nc], dtype=np.int32)


def write_input_params_ess(path, nu0: float, dnu: float, chan0: float, data_path: str) -> None:
    with open(path, "w") as f:
        f.write(f"{nu0!r}\t{dnu!r}\t{chan0!r}\t{data_path}\n")


def read_input_params_ess(path):
    with open(path) as f:
        tok = f.read().split()
    return float(tok[0]), float(tok[1]), float(tok[2]), tok[3]


def write_rings_file(path, ulow, uhigh) -> None:
    """Ring edges for the reference harness: Nr, then 'ULow UHigh' per line,
    with 17 significant digits so the edges round-trip exactly."""
    with open(path, "w") as f:
        f.write(f"{len(ulow)}\n")
        for lo, hi in zip(ulow, uhigh):
            f.write(f"{float(lo):.17g} {float(hi):.17g}\n")


def read_closed_rings(res_path):
    with open(os.path.join(res_path, "rcount")) as f:
        rcount = int(f.read().split()[0])
    data = np.fromfile(os.path.join(res_path, "closed_rings"), dtype=np.float64, count=4 * rcount)
    return data.reshape(rcount, 4)


def write_closed_rings(res_path, rdata: np.ndarray) -> None:
    os.makedirs(res_path, exist_ok=True)
    np.ascontiguousarray(rdata, dtype=np.float64).tofile(os.path.join(res_path, "closed_rings"))
    with open(os.path.join(res_path, "rcount"), "w") as f:
        f.write(f"{rdata.shape[0]}")


def bsout_name(version: int, r1: int, r2: int, r3: int, rlzn: int) -> str:
    stem = "bsout_final" if version == 1 else "bsout_final2"
    return f"{stem}_ra{r1}_rb{r2}_rc{r3}_R{rlzn}"


def write_bsout_v1(path, ntri: float, num: float, bldnu: np.ndarray, numdnu: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<dd", ntri, num))
        np.ascontiguousarray(bldnu, dtype=np.float32).tofile(f)
        np.ascontiguousarray(numdnu, dtype=np.int32).tofile(f)


def write_bsout_v2(path, inv_ng1_ng2: float, bldnu: np.ndarray, numdnu: np.ndarray) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<d", inv_ng1_ng2))
        np.ascontiguousarray(bldnu, dtype=np.float32).tofile(f)
        np.ascontiguousarray(numdnu, dtype=np.float32).tofile(f)


def read_bsout_v1(path, nclen: int, bl_dtype=np.float32):
    """Raw v1 record: (Ntri, Num, bldnu[nclen,nclen], numdnu int32[nclen,nclen]).
    ``bl_dtype=np.float64`` reads the FP64 reference build's files."""
    n = nclen * nclen
    with open(path, "rb") as f:
        ntri, num = struct.unpack("<dd", f.read(16))
        bl = np.fromfile(f, dtype=bl_dtype, count=n)
        nd = np.fromfile(f, dtype=np.int32, count=n)
    return ntri, num, bl.reshape(nclen, nclen), nd.reshape(nclen, nclen)


def read_bsout_v2(path, nclen: int, dtype=np.float32):
    n = nclen * nclen
    with open(path, "rb") as f:
        (inv,) = struct.unpack("<d", f.read(8))
        bl = np.fromfile(f, dtype=dtype, count=n)
        nd = np.fromfile(f, dtype=dtype, count=n)
    return inv, bl.reshape(nclen, nclen), nd.reshape(nclen, nclen)


VIS_MAGIC = b"AMBRVIS1"
VIS_HEADER = struct.Struct("<8sqqqqffff")


def write_vis(path, randpar: np.ndarray, data: np.ndarray, nu_chan0: float, del_chan: float, chan0: float) -> None:
    """Synthetic stand-in for a random-groups UVFITS file: randpar float32
    [G, pcount] (u/ν0, v/ν0, ...), data float32 [G, nchan, nstokes, 3]."""
    g, pcount = randpar.shape
    _, nchan, nstokes, three = data.shape
    assert three == 3 and data.shape[0] == g
    with open(path, "wb") as f:
        f.write(VIS_HEADER.pack(VIS_MAGIC, g, pcount, nstokes, nchan, nu_chan0, del_chan, chan0, 0.0))
        rec = np.concatenate(
            [randpar.astype(np.float32), data.astype(np.float32).reshape(g, -1)], axis=1
        )
        rec.tofile(f)


def write_cldnu(path, cldnu: np.ndarray, numdnu: np.ndarray, binu: np.ndarray, num: np.ndarray) -> None:
    """MAPS result file (4_fbe/maps.c:195-206): for every bin i and channel lag j one line
    "i\tbinu[i]\tj\tcldnu[i][j]\tnumdnu[j]\tnum[i]" with C's %e for the reals."""
    nb, nc = cldnu.shape
    with open(path, "w") as f:
        for i in range(nb):
            for j in range(nc):
                f.write(f"{i}\t{binu[i]:e}\t{j}\t{cldnu[i, j]:e}\t{numdnu[j]:e}\t{int(num[i])}\n")


def read_cldnu(path):
    """Parse a MAPS result file: (cldnu [nb, nc], numdnu [nc], binu [nb], num [nb]) at the
    file's printed precision."""
    rows = [ln.split("\t") for ln in open(path).read().splitlines() if ln.strip()]
    nb = max(int(r[0]) for r in rows) + 1
    nc = max(int(r[2]) for r in rows) + 1
    cl, nd = np.zeros((nb, nc)), np.zeros(nc)
    bu, nm = np.zeros(nb), np.zeros(nb, dtype=np.int64)
    for r in rows:
        i, j = int(r[0]), int(r[2])
        bu[i], cl[i, j], nd[j], nm[i] = float(r[1]), float(r[3]), float(r[4]), int(r[5])
    return cl, nd, bu, nm
