"""Generates the golden fixtures in this directory by running the MorphStore
reference's own codecs and operators (AVX-512 build of oracle/ref_shim.cpp,
compiled from the reference source tree by oracle/Makefile).

    make -C oracle ref && python tests/golden/make_golden.py

Inputs come from the oracle's seeded generators; outputs (compressed bytes,
column metadata, positions, group ids, sums) come from the reference.  The
fixtures pin the C oracle (tests/test_golden_cpu.py) and the CUDA path
(tests/test_golden_gpu.py) without needing the reference at test time.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from oracle import selector_ref as SR  # noqa: E402

OUT = os.path.join(HERE, "golden.npz")


def inputs(orc):
    """Named seeded input columns of the four distributions and odd lengths."""
    geo4 = orc.geom_table(0.25)
    zipf = orc.zipf_table(1.2, 1 << 20)
    cols = {}
    for n in (17, 1234, 4096 + 17, 33_000 + 9):
        cols[f"uni20_{n}"] = orc.uniform_bits(n, 20, n)
        cols[f"zipf_{n}"] = orc.from_table(n + 1, zipf, n)
        cols[f"sorted_{n}"] = orc.sorted_gaps(n + 2, geo4, n)
        cols[f"runs_{n}"] = orc.runs(n + 3, 5, 20, n)
    cols["uni64_9000"] = orc.uniform_bits(64, 64, 9000)
    cols["uni12_40077"] = orc.uniform_bits(12, 12, 40_077)
    return cols


def bwi_inputs(orc):
    """96 blocks of 2048 values (uniform over 1..64 bits, sorted with gaps,
    runs, Zipf, constant), one pick per block cycling through static_vbp,
    dynamic_vbp, delta+dvbp and for+dvbp (the formats the reference's
    container and the GPU's share), and the format codes of those picks."""
    from oracle import selector_ref as SR
    geo, zipf = orc.geom_table(0.25), orc.zipf_table(1.2, 1 << 20)
    blocks = []
    for i in range(96):
        kind = i % 6
        if kind == 0:
            blocks.append(orc.uniform_bits(700 + i, 1 + (i * 7) % 64, 2048))
        elif kind == 1:
            blocks.append(orc.sorted_gaps(700 + i, geo, 2048) + np.uint64(i << 30))
        elif kind == 2:
            blocks.append(orc.runs(700 + i, 5, 20, 2048))
        elif kind == 3:
            blocks.append(orc.from_table(700 + i, zipf, 2048))
        elif kind == 4:
            blocks.append(np.full(2048, i * 977, dtype=np.uint64))
        else:
            blocks.append(orc.uniform_bits(700 + i, 12, 2048) + np.uint64(1 << 40))
    x = np.concatenate(blocks)
    choice = np.array([(i * 5 + i // 4) % 4 for i in range(96)], dtype=np.uint8)
    codes = np.array([SR.candidate_payload(orc, x[b * 2048:(b + 1) * 2048], int(choice[b]))[0] for b in range(96)],
                     dtype=np.uint8)
    return x, choice, codes


def main():
    path = O.reference_path("avx512")
    if path is None:
        raise SystemExit("build the reference first: make -C oracle ref")
    ref = O.Reference(path)
    orc = O.Oracle()
    cols = inputs(orc)
    fx = {}
    for name, v in cols.items():
        fx[f"in/{name}"] = v
    # --- codecs ---------------------------------------------------------------
    for name, v in cols.items():
        fmts = [(O.DYNAMIC_VBP, 0), (O.DELTA_DVBP, 0), (O.FOR_DVBP, 0), (O.RLE, 0)]
        if name.startswith("uni20"):
            fmts += [(O.STATIC_VBP, 20), (O.STATIC_VBP, 33)]
        if name == "uni64_9000":
            fmts = [(O.STATIC_VBP, 64), (O.DYNAMIC_VBP, 0), (O.FOR_DVBP, 0), (O.DELTA_DVBP, 0)]
        for fmt, bw in fmts:
            b, m = ref.compress(fmt, bw, v)
            key = f"codec/{name}/{fmt}/{bw}"
            fx[key + "/bytes"] = O.mask_gap(fmt, bw, b, m, orc)
            fx[key + "/meta"] = np.array(m, dtype=np.uint64)
    for bw in range(1, 65):
        v = orc.uniform_bits(1000 + bw, bw, 1024 + 37)
        b, m = ref.compress(O.STATIC_VBP, bw, v)
        fx[f"static/{bw}/in"] = v
        fx[f"static/{bw}/bytes"] = O.mask_gap(O.STATIC_VBP, bw, b, m, orc)
        fx[f"static/{bw}/meta"] = np.array(m, dtype=np.uint64)
    # --- select with compressed inputs / outputs ----------------------------------
    x = cols["uni12_40077"]
    for in_fmt, in_bw in [(O.UNCOMPR, 0), (O.DYNAMIC_VBP, 0), (O.DELTA_DVBP, 0), (O.FOR_DVBP, 0)]:
        if in_fmt == O.UNCOMPR:
            xb, xm = x.view(np.uint8).copy(), (len(x), 8 * len(x), 0)
        else:
            xb, xm = ref.compress(in_fmt, in_bw, x)
        for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
            ob, om = ref.select(O.CMP_LT, 1500, in_fmt, in_bw, xb, xm, out_fmt, 0)
            key = f"select/{in_fmt}/{out_fmt}"
            fx[key + "/bytes"] = O.mask_gap(out_fmt, 0, ob, om, orc)
            fx[key + "/meta"] = np.array(om, dtype=np.uint64)
    for cmp in range(5):
        ob, om = ref.select(cmp, 2048, O.UNCOMPR, 0, x.view(np.uint8), (len(x), 8 * len(x), 0), O.UNCOMPR, 0)
        fx[f"select_cmp/{cmp}"] = ob.view(np.uint64)
    # --- select on values >= 2^63 (AVX-512 signed compare) -------------------------
    w = cols["uni64_9000"]
    ob, om = ref.select(O.CMP_LT, 1 << 62, O.UNCOMPR, 0, w.view(np.uint8), (len(w), 8 * len(w), 0), O.UNCOMPR, 0)
    fx["select_signed"] = ob.view(np.uint64)
    # --- project --------------------------------------------------------------------
    y = cols["uni20_33009"]
    yb, ym = ref.compress(O.STATIC_VBP, 20, y)
    pos = np.arange(3, len(y), 7, dtype=np.uint64)
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP):
        ob, om = ref.project(O.STATIC_VBP, 20, yb, ym, O.UNCOMPR, 0, pos.view(np.uint8), (len(pos), 8 * len(pos), 0),
                             out_fmt, 0)
        fx[f"project/{out_fmt}/bytes"] = O.mask_gap(out_fmt, 0, ob, om, orc)
        fx[f"project/{out_fmt}/meta"] = np.array(om, dtype=np.uint64)
    # --- agg_sum ----------------------------------------------------------------------
    for fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP, O.FOR_DVBP):
        v = cols["sorted_33009"]
        if fmt == O.UNCOMPR:
            s = ref.agg_sum(fmt, 0, v.view(np.uint8), (len(v), 8 * len(v), 0))
        else:
            b, m = ref.compress(fmt, 0, v)
            s = ref.agg_sum(fmt, 0, b, m)
        fx[f"agg_sum/{fmt}"] = np.array([s], dtype=np.uint64)
    # --- semi_join ----------------------------------------------------------------------
    dim = orc.sorted_gaps(5, orc.geom_table(0.25), 3000)
    keep = orc.uniform_bits(6, 4, len(dim)) < 2
    lkeys = dim[keep]
    fk = orc.uniform_bits(7, 14, 30_011)
    fx["semi/l"] = lkeys
    fx["semi/r"] = fk
    lb, lm = ref.compress(O.DELTA_DVBP, 0, lkeys)
    rb, rm = ref.compress(O.FOR_DVBP, 0, fk)
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP, O.DELTA_DVBP):
        ob, om = ref.semi_join(O.DELTA_DVBP, lb, lm, O.FOR_DVBP, rb, rm, out_fmt)
        fx[f"semi/{out_fmt}/bytes"] = O.mask_gap(out_fmt, 0, ob, om, orc)
        fx[f"semi/{out_fmt}/meta"] = np.array(om, dtype=np.uint64)
    # --- natural equi-join (duplicate build keys: the first position wins) -------------------
    lk = orc.uniform_bits(12, 11, 4000)
    rk = orc.uniform_bits(13, 12, 30_011)
    fx["njoin/l"], fx["njoin/r"] = lk, rk
    lb, lm = ref.compress(O.DELTA_DVBP, 0, lk)
    rb, rm = ref.compress(O.FOR_DVBP, 0, rk)
    for out_fmt in (O.UNCOMPR, O.DYNAMIC_VBP):
        (ob, om), (pb, pm) = ref.natural_join(O.DELTA_DVBP, lb, lm, O.FOR_DVBP, rb, rm, out_fmt)
        fx[f"njoin/{out_fmt}/l/bytes"] = O.mask_gap(out_fmt, 0, ob, om, orc)
        fx[f"njoin/{out_fmt}/l/meta"] = np.array(om, dtype=np.uint64)
        fx[f"njoin/{out_fmt}/r/bytes"] = O.mask_gap(out_fmt, 0, pb, pm, orc)
        fx[f"njoin/{out_fmt}/r/meta"] = np.array(pm, dtype=np.uint64)
    # --- intersect -----------------------------------------------------------------------
    a = np.flatnonzero(orc.uniform_bits(8, 3, 20_000) < 3).astype(np.uint64)
    b2 = np.flatnonzero(orc.uniform_bits(9, 3, 20_000) < 5).astype(np.uint64)
    fx["isect/l"], fx["isect/r"] = a, b2
    # the scalar intersect_sorted: the vectorised my_intersect_wit_t crashes
    # (segmentation fault) in this build on uncompressed and dynamic_vbp inputs
    fx["isect/out"] = ref.intersect_scalar(a, b2)
    # --- group + grouped sum ---------------------------------------------------------------
    g = orc.from_table(10, orc.zipf_table(1.1, 1000), 50_003)
    meas = orc.uniform_bits(11, 16, len(g))
    fx["group/in"], fx["group/meas"] = g, meas
    gb, gm = ref.compress(O.DYNAMIC_VBP, 0, g)
    (grb, grm), (exb, exm) = ref.group(O.DYNAMIC_VBP, gb, gm, O.UNCOMPR, O.UNCOMPR)
    fx["group/gr"] = grb.view(np.uint64)
    fx["group/ext"] = exb.view(np.uint64)
    (grb2, grm2), (exb2, exm2) = ref.group(O.DYNAMIC_VBP, gb, gm, O.DYNAMIC_VBP, O.DYNAMIC_VBP)
    fx["group/gr_dvbp/bytes"] = O.mask_gap(O.DYNAMIC_VBP, 0, grb2, grm2, orc)
    fx["group/gr_dvbp/meta"] = np.array(grm2, dtype=np.uint64)
    fx["group/ext_dvbp/bytes"] = O.mask_gap(O.DYNAMIC_VBP, 0, exb2, exm2, orc)
    fx["group/ext_dvbp/meta"] = np.array(exm2, dtype=np.uint64)
    fx["group/sum"] = ref.agg_sum_grouped(fx["group/gr"], meas, len(fx["group/ext"]))
    # --- blockwise_individual_f and the exhaustive selector (ref_bwi.cpp) -------------------
    x, choice, codes = bwi_inputs(orc)
    fx["bwi/in"], fx["bwi/choice"], fx["bwi/codes"] = x, choice, codes
    fx["bwi/bytes"] = SR.mask_container(ref.bwi_compress(x, codes), choice)
    fx["bwi/exhaustive"] = ref.exhaustive_choose(x)
    np.savez_compressed(OUT, **fx)
    print(f"wrote {OUT}: {len(fx)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
