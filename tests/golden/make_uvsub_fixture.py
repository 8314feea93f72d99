"""Generate tests/golden/uvsub_fixture.npz from the reference's own golden test
of the DFT path, Obit/testScripts/testUVSub.py (reference paths below are within
ObitSystem/Obit of the reference tree):

  input   testData/UVSubTestIn.uvtab       15949 records, RR LL RL LR, 1 ch x 2 IF
  model   testData/UVSubTestModIn.fits.gz  CC table version 2 (13 components)
  master  testData/UVSubTestMaster.uvtab   the script's expected output

The script divides the DFT of the CC model into the data (SkyModel.PDivUV with
Mode=DFT, Factor=0.5, Stokes '    ', CCVer=2, do3D False) using a mosaic that
holds the same image twice, so every component enters twice at half flux, and
reports ObitUVUtilVisCompare(out, master), a fractional RMS it does not assert.

This script restates, in numpy, what the reference does before the DFT:
  * component positions, ObitSkyModelLoadComps (src/ObitSkyModel.c:1888-1989):
    field offset from ObitUVDescShiftPhase -> ObitSkyGeomShiftSIN
    (src/ObitUVDesc.c:735-790, src/ObitSkyGeom.c:177-205), rotation terms from
    ObitImageDescRotate / ObitUVDescRotate, and the 3-D re-projection matrix of
    ObitUVDescShift3DMatrix (src/ObitUVDesc.c:882-978; the image carries no DO3D
    key, so it is a 3-D image, src/ObitIOImageFITS.c:2053-2059), with the
    reference's FP32 (ofloat) rounding points;
  * channel frequencies: FREQ CRVAL plus the FQ table's IF offsets
    (ObitUVDescGetFreq, src/ObitUVDesc.c:506-617);
  * polarizations: Stokes '    ' on RR,LL,RL,LR data models the first two
    (src/ObitSkyModel.c:3743, 3805-3823) with stokFactor 1;
and then runs the FP64 oracle's divide and the metric of
ObitUVUtilVisCompare (src/ObitUVUtil.c:1350-1506, restated in vis_compare).

Only this generator reads the reference tree; the committed fixture holds a
row subset (every STRIDE-th record) of input and master, the component table,
the CC rows and image / uv geometry it came from, the frequencies, and the
full-data RMS values measured here.

Run:  python tests/golden/make_uvsub_fixture.py [path/to/ObitSystem/Obit]
"""
from __future__ import annotations

import gzip
import json
import math
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path[:0] = [str(ROOT), str(ROOT / "oracle"), str(ROOT / "tests")]

DG2RAD = math.pi / 180.0
STRIDE = 8
F32 = np.float32


# ---- minimal FITS reading ------------------------------------------------------


def _hdus(raw: bytes):
    """Yield (cards dict, data bytes) for each HDU of a FITS byte string."""
    off = 0
    while off < len(raw):
        cards, done = {}, False
        while not done:
            blk = raw[off:off + 2880]
            off += 2880
            for i in range(36):
                c = blk[i * 80:(i + 1) * 80].decode("ascii", "replace")
                if c.startswith("END") and c[3:].strip() == "":
                    done = True
                    break
                if c[8:10] == "= ":
                    v = c[10:]
                    if v.strip().startswith("'"):
                        v = v.strip()[1:].split("'")[0].rstrip()
                    else:
                        v = v.split("/")[0].strip()
                    cards[c[:8].strip()] = v
        n = 0
        if int(cards.get("NAXIS", 0)) > 0:
            n = abs(int(cards["BITPIX"])) // 8
            for i in range(1, int(cards["NAXIS"]) + 1):
                n *= int(cards[f"NAXIS{i}"])
            n += int(cards.get("PCOUNT", 0))
        yield cards, raw[off:off + n]
        off += (n + 2879) // 2880 * 2880


def _table(cards, data):
    """Columns of a binary table as big-endian numpy arrays, by TTYPE."""
    codes = {"E": ">f4", "D": ">f8", "J": ">i4", "I": ">i2", "A": "S1", "L": "S1", "B": "u1"}
    fields, width = [], 0
    for i in range(1, int(cards["TFIELDS"]) + 1):
        form = cards[f"TFORM{i}"].strip()
        rep = int(form[:-1] or 1)
        code = form[-1]
        fields.append((cards[f"TTYPE{i}"].strip(), codes[code], rep))
    dt = np.dtype([(n, c, (r,)) if r > 1 and c != "S1" else (n, f"S{r}" if c == "S1" else c)
                   for n, c, r in fields])
    assert dt.itemsize == int(cards["NAXIS1"])
    return np.frombuffer(data, dtype=dt, count=int(cards["NAXIS2"]))


def read_uvtab(path: Path):
    raw = path.read_bytes()
    hd = list(_hdus(raw))
    uv = next((c, d) for c, d in hd if c.get("EXTNAME") == "AIPS UV")
    fq = next((c, d) for c, d in hd if c.get("EXTNAME") == "AIPS FQ")
    t = _table(*uv)
    cards = uv[0]
    tdim = [int(x) for x in cards["TDIM6"].strip("()").split(",")]
    ncorr = tdim[1] * tdim[2] * tdim[3]
    nrparm = 5
    rec = np.empty((len(t), nrparm + 3 * ncorr), np.float32)
    # random parameters are stored in wavelengths at the reference frequency
    # (TSCAL = 1/freq converts them to seconds); Obit uses the stored values
    rec[:, 0] = t["UU---SIN"]
    rec[:, 1] = t["VV---SIN"]
    rec[:, 2] = t["WW---SIN"]
    rec[:, 3] = t["BASELINE"]
    rec[:, 4] = t["DATE"]
    rec[:, nrparm:] = t["VISIBILITIES"].astype(np.float32)
    fqt = _table(*fq)
    iffreq = np.asarray(fqt["IF FREQ"][0], np.float64)
    ref = float(cards["3CRVL6"])
    axes = {"nstok": tdim[1], "nchan": tdim[2], "nif": tdim[3],
            "crval_stokes": float(cards["2CRVL6"]), "ref_freq": ref,
            "ra": float(cards["5CRVL6"]), "dec": float(cards["6CRVL6"]),
            "uvrot": float(cards.get("6CROT6", 0.0))}
    assert tdim[0] == 3 and tdim[2] == 1
    freq_arr = ref + iffreq                    # one channel per IF, CRPIX 1
    return rec, freq_arr, axes


def read_model(path: Path, ccver: int = 2):
    raw = gzip.open(path, "rb").read()
    hd = list(_hdus(raw))
    img = hd[0][0]
    cc = [(c, d) for c, d in hd if c.get("EXTNAME") == "AIPS CC" and int(c["EXTVER"]) == ccver]
    t = _table(*cc[0])
    desc = {"ra": float(img["CRVAL1"]), "dec": float(img["CRVAL2"]),
            "rot": float(img.get("CROTA2", 0.0)), "ctype": img["CTYPE1"],
            "do3D": "DO3D" not in img or int(img["DO3D"]) == 2,
            "xPxOff": float(img.get("XPXOFF", 0.0)), "yPxOff": float(img.get("YPXOFF", 0.0)),
            "cdelt": (float(img["CDELT1"]), float(img["CDELT2"]))}
    return np.stack([t["FLUX"], t["DELTAX"], t["DELTAY"]], axis=1).astype(np.float32), desc


# ---- component positions (ObitSkyModelLoadComps) ------------------------------


def shift_sin(ra, dec, rotate, xra, xdec):
    """ObitSkyGeomShiftSIN: FP64 direction cosines, FP32 results.  (The
    reference's DG2RAD macro expands unparenthesized: rotate * pi / 180.)"""
    maprr = F32(float(F32(rotate)) * math.pi / 180.0)
    xx = math.cos(DG2RAD * xdec) * math.sin(DG2RAD * (xra - ra))
    yy = (math.sin(DG2RAD * xdec) * math.cos(DG2RAD * dec)
          - math.cos(DG2RAD * xdec) * math.sin(DG2RAD * dec) * math.cos(DG2RAD * (xra - ra)))
    xs = F32(math.cos(maprr) * xx + math.sin(maprr) * yy)
    ys = F32(-math.sin(maprr) * xx + math.cos(maprr) * yy)
    dz = math.sqrt(1.0 - float(xs * xs) - float(ys * ys))  # FP32 squares
    return np.array([2.0 * math.pi * float(xs), 2.0 * math.pi * float(ys),
                     2.0 * math.pi * (dz - 1.0)], dtype=np.float32)


def urot3d(ra, dec, xra, xdec, mrot, urot):
    """ObitUVDescShift3DMatrix, 3-D image branch: U = R(map+) X R(uv-)."""
    sa, ca = math.sin(DG2RAD * (xra - ra)), math.cos(DG2RAD * (xra - ra))
    sd, cd = math.sin(DG2RAD * xdec), math.cos(DG2RAD * xdec)
    sd0, cd0 = math.sin(DG2RAD * dec), math.cos(DG2RAD * dec)
    r = DG2RAD * float(F32(mrot))
    rmap = np.array([[math.cos(r), math.sin(r), 0.0], [-math.sin(r), math.cos(r), 0.0],
                     [0.0, 0.0, 1.0]])
    x = np.array([[ca, sd0 * sa, -cd0 * sa],
                  [-sd * sa, cd * cd0 + sd * sd0 * ca, cd * sd0 - sd * cd0 * ca],
                  [cd * sa, sd * cd0 - cd * sd0 * ca, sd * sd0 + cd * cd0 * ca]])
    r = DG2RAD * float(F32(urot))
    ruv = np.array([[math.cos(r), -math.sin(r), 0.0], [math.sin(r), math.cos(r), 0.0],
                    [0.0, 0.0, 1.0]])
    # t[j][i] = sum_k x[k][i] rm[j][k]; U[j][i] = sum_k ruv[k][i] t[j][k], in
    # the reference's summation order
    t = [[sum_ordered(x[k][i] * rmap[j][k] for k in range(3)) for i in range(3)] for j in range(3)]
    u = [[sum_ordered(ruv[k][i] * t[j][k] for k in range(3)) for i in range(3)] for j in range(3)]
    return np.array(u).astype(np.float32)


def sum_ordered(terms):
    acc = 0.0
    for v in terms:
        acc += v
    return acc


def load_comps(cc, img, uv_axes, factor, do3D_model, nfield):
    """Component table [flux, X, Y, Z] of `nfield` copies of one image's CCs."""
    konst = F32(DG2RAD * 2.0 * math.pi)
    maprot, uvrot = F32(img["rot"]), F32(uv_axes["uvrot"])
    ssrot = F32(math.sin(DG2RAD * float(F32(uvrot - maprot))))
    ccrot = F32(math.cos(DG2RAD * float(F32(uvrot - maprot))))
    assert img["do3D"], "2-D image geometry is not restated"
    assert img["ctype"][4:8] == "-SIN"
    dxyzc = shift_sin(uv_axes["ra"], uv_axes["dec"], maprot, img["ra"], img["dec"])
    if do3D_model:
        xpoff = ypoff = F32(0.0)
    else:
        xpoff = F32(img["xPxOff"]) * F32(img["cdelt"][0])
        ypoff = F32(img["yPxOff"]) * F32(img["cdelt"][1])
    xxoff = F32(dxyzc[0] * ccrot + dxyzc[1] * ssrot)
    yyoff = F32(dxyzc[1] * ccrot - dxyzc[0] * ssrot)
    zzoff = dxyzc[2]
    do3Dmul = (maprot != 0 or uvrot != 0 or abs(img["ra"] - uv_axes["ra"]) > 1e-10
               or abs(img["dec"] - uv_axes["dec"]) > 1e-10 or img["xPxOff"] != 0
               or img["yPxOff"] != 0)
    U = urot3d(uv_axes["ra"], uv_axes["dec"], img["ra"], img["dec"], maprot, uvrot)
    # ObitTableCCUtilMergeSel merges equal positions; the table is already merged
    assert len({(float(a), float(b)) for _, a, b in cc}) == len(cc)
    rows = []
    for _ in range(nfield):
        for flux, dx, dy in cc:
            xp0 = F32(F32(dx + xpoff) * konst)
            xp1 = F32(F32(dy + ypoff) * konst)
            if do3Dmul:
                xyz = [F32(xp0 * U[0, c] + xp1 * U[1, c]) for c in range(3)]
            else:
                xyz = [F32(ccrot * xp0 + ssrot * xp1), F32(ccrot * xp1 - ssrot * xp0), F32(0.0)]
            rows.append([F32(flux * F32(factor)), F32(xyz[0] + xxoff), F32(xyz[1] + yyoff),
                         F32(xyz[2] + zzoff)])
    return np.array(rows, np.float32)


def vis_compare(a, b, nrparm):
    """ObitUVUtilVisCompare metric (src/ObitUVUtil.c:1455-1503)."""
    x = a[:, nrparm:].reshape(len(a), -1, 3).astype(np.float64)
    y = b[:, nrparm:].reshape(len(b), -1, 3).astype(np.float64)
    amp = np.sqrt(y[..., 0] ** 2 + y[..., 1] ** 2)
    ok = (x[..., 2] > 0) & (y[..., 2] > 0) & (amp > 0)
    s = ((x[..., 0] - y[..., 0]) ** 2 + (x[..., 1] - y[..., 1]) ** 2)[ok] / amp[ok]
    return float(math.sqrt(s.sum() / (2 * ok.sum())))


def main():
    # the reference's ObitSystem/Obit directory: the first argument, else
    # $OBIT_REFERENCE/ObitSystem/Obit, else the reference checked out beside
    # this repository (../reference)
    if len(sys.argv) > 1:
        ref = Path(sys.argv[1])
    else:
        root = os.environ.get("OBIT_REFERENCE") or str(Path(__file__).resolve().parents[3] / "reference")
        ref = Path(root) / "ObitSystem" / "Obit"
    td = ref / "testData"
    rec, freq_arr, axes = read_uvtab(td / "UVSubTestIn.uvtab")
    master, _, _ = read_uvtab(td / "UVSubTestMaster.uvtab")
    cc, img = read_model(td / "UVSubTestModIn.fits.gz")
    comps = load_comps(cc, img, axes, factor=0.5, do3D_model=False, nfield=2)

    import oracle
    from obit_b200 import uvdata as U
    from obit_b200.skymodel import OP_DIV, SkyModelParams

    uv = U.UVData(rec, axes["nstok"], axes["nchan"], axes["nif"], axes["ref_freq"], freq_arr,
                  crval_stokes=axes["crval_stokes"])
    sky = U.SkyComps(U.MOD_POINT, comps)
    p = SkyModelParams(op=OP_DIV, startPoln=1, numberPoln=2)
    out = oracle.apply_fp64(uv, sky, p)
    rms_in = vis_compare(rec, master, 5)
    rms_fp64 = vis_compare(out, master, 5)
    info = {"records": int(len(rec)), "stride": STRIDE, "components": int(len(comps)),
            "ref_freq": axes["ref_freq"], "freq_arr": [float(f) for f in freq_arr],
            "visCompare_input_vs_master": rms_in,
            "visCompare_fp64_oracle_vs_master": rms_fp64}
    if oracle.have_refcpu():
        info["visCompare_refcpu_vs_master"] = vis_compare(oracle.apply_refcpu(uv, sky, p), master, 5)
    sub = slice(0, None, STRIDE)
    np.savez_compressed(HERE / "uvsub_fixture.npz", input=rec[sub], master=master[sub],
                        comps=comps, freq_arr=freq_arr,
                        axes=np.array([axes["nstok"], axes["nchan"], axes["nif"]], np.int32),
                        ref_freq=np.float64(axes["ref_freq"]),
                        crval_stokes=np.float64(axes["crval_stokes"]),
                        # the CC rows and geometry the component table came from
                        cc=cc, cc_factor=np.float32(0.5), cc_nfield=np.int32(2),
                        im_geom=np.array([img["ra"], img["dec"], img["rot"], float(img["do3D"]),
                                          img["xPxOff"], img["yPxOff"], img["cdelt"][0],
                                          img["cdelt"][1]], np.float64),
                        uv_geom=np.array([axes["ra"], axes["dec"], axes["uvrot"]], np.float64))
    (HERE / "uvsub_fixture.json").write_text(json.dumps(info, indent=1) + "\n")
    print(json.dumps(info, indent=1))


if __name__ == "__main__":
    main()
