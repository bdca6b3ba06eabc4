"""Golden fixtures for histio.py from the reference's own histogram I/O.

Writes small seeded PGM / PPM images and a CSV column, loads them with the
reference's load_img_to_pdf, load_rgb_img_to_pdf_grayscale_luma,
load_img_to_pdf_gamma_correction and load_csv_to_pdf (cpp/histogramIO.h:243-337,
compiled by oracle/Makefile into oracle/_ref/libhistioref.so; CImg reads PNM
natively), exports histograms with save_pdf / save_pdf_gamma_correction
(:339-371) and evaluates quantile (:379-405).  The input files' bytes and the
outputs go to histio_ref.npz.

    python tests/golden/make_golden_histio.py
"""
from __future__ import annotations

import ctypes as C
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(ROOT, "oracle", "_ref", "libhistioref.so")

_dp = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


def main():
    L = C.CDLL(REF)
    for name in ("href_load_img_to_pdf", "href_load_rgb_luma"):
        getattr(L, name).restype = C.c_double
        getattr(L, name).argtypes = [C.c_char_p, _dp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.href_load_gamma.restype = C.c_double
    L.href_load_gamma.argtypes = [C.c_char_p, _dp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_double,
                                  C.c_int]
    L.href_load_csv.restype = C.c_int
    L.href_load_csv.argtypes = [C.c_char_p, _dp, C.c_int, _dp]
    L.href_save_pdf.argtypes = [C.c_char_p, C.c_int, C.c_int, _dp, C.c_double]
    L.href_save_pdf_gamma.argtypes = [C.c_char_p, C.c_int, C.c_int, _dp, C.c_double, C.c_int, C.c_double]
    L.href_quantile.argtypes = [_dp, C.c_int, _dp, C.c_int, _dp]

    rng = np.random.Generator(np.random.PCG64(4321))
    W, H = 13, 9
    gray = rng.integers(0, 256, (H, W)).astype(np.uint8)
    rgb = rng.integers(0, 256, (H, W, 3)).astype(np.uint8)
    pgm = b"P5\n%d %d\n255\n" % (W, H) + gray.tobytes()
    ppm = b"P6\n%d %d\n255\n" % (W, H) + rgb.tobytes()
    csv_vals = rng.random(17) * 3.0
    csv = "".join("%.17g\n" % v for v in csv_vals).encode()
    out = dict(W=W, H=H, pgm=np.frombuffer(pgm, np.uint8), ppm=np.frombuffer(ppm, np.uint8),
               csv=np.frombuffer(csv, np.uint8))
    with tempfile.TemporaryDirectory() as d:
        paths = {}
        for key, data in (("pgm", pgm), ("ppm", ppm), ("csv", csv)):
            paths[key] = os.path.join(d, "in." + key)
            open(paths[key], "wb").write(data)
        w, h = C.c_int(), C.c_int()
        buf = np.zeros(W * H)
        out["sum_gray"] = L.href_load_img_to_pdf(paths["pgm"].encode(), _p(buf), buf.size, C.byref(w), C.byref(h))
        out["pdf_gray"] = buf.copy()
        out["sum_ppm_first"] = L.href_load_img_to_pdf(paths["ppm"].encode(), _p(buf), buf.size, C.byref(w),
                                                      C.byref(h))
        out["pdf_ppm_first"] = buf.copy()
        out["sum_luma"] = L.href_load_rgb_luma(paths["ppm"].encode(), _p(buf), buf.size, C.byref(w), C.byref(h))
        out["pdf_luma"] = buf.copy()
        for alpha, comp in ((0.5, 0), (2.2, 1)):
            s = L.href_load_gamma(paths["pgm"].encode(), _p(buf), buf.size, C.byref(w), C.byref(h), alpha, comp)
            out[f"sum_gamma_{alpha}_{comp}"] = s
            out[f"pdf_gamma_{alpha}_{comp}"] = buf.copy()
        cbuf = np.zeros(64)
        csum = C.c_double()
        n = L.href_load_csv(paths["csv"].encode(), _p(cbuf), cbuf.size, C.byref(csum))
        out["pdf_csv"] = cbuf[:n].copy()
        out["sum_csv"] = csum.value
        # exporters: the gray pdf scaled back to 0..255-ish values, and gamma-corrected
        val = np.ascontiguousarray(out["pdf_gray"])
        scaling = 255.0 / float(val.max())
        p1 = os.path.join(d, "out1.ppm")
        L.href_save_pdf(p1.encode(), W, H, _p(val), scaling)
        out["save_pdf_scaling"] = scaling
        out["save_pdf_bytes"] = np.frombuffer(open(p1, "rb").read(), np.uint8)
        p2 = os.path.join(d, "out2.ppm")
        L.href_save_pdf_gamma(p2.encode(), W, H, _p(val), 2.2, 1, 1.0 / float(val.max()))
        out["save_gamma_scaling"] = 1.0 / float(val.max())
        out["save_gamma_bytes"] = np.frombuffer(open(p2, "rb").read(), np.uint8)
    data = rng.random(50)
    probs = np.array([0.0, 0.1, 0.25, 0.5, 0.9, 1.0])
    q = np.zeros(probs.size)
    L.href_quantile(_p(data), data.size, _p(probs), probs.size, _p(q))
    out.update(quantile_data=data, quantile_probs=probs, quantile=q)
    path = os.path.join(HERE, "histio_ref.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    sys.exit(main())
