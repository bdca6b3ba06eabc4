"""Histogram I/O (no GPU): PNM / PNG readers and writers, the reference's
image-to-histogram conversions and exporters (cpp/histogramIO.h)."""
import os

import numpy as np
import pytest

from wassersteindictionarylearning_b200 import histio as hio


@pytest.fixture
def img():
    rng = np.random.default_rng(3)
    return rng.integers(0, 256, size=(37, 53)).astype(np.uint8)


@pytest.mark.parametrize("ext", [".pgm", ".png"])
def test_grey_round_trip(tmp_path, img, ext):
    p = str(tmp_path / ("a" + ext))
    hio.write_image(p, img)
    back = hio.read_image(p)
    assert back.shape == img.shape and np.array_equal(back, img.astype(np.float64))


@pytest.mark.parametrize("ext", [".ppm", ".png"])
def test_rgb_round_trip(tmp_path, ext):
    rgb = np.random.default_rng(4).integers(0, 256, size=(20, 31, 3)).astype(np.uint8)
    p = str(tmp_path / ("b" + ext))
    hio.write_image(p, rgb)
    assert np.array_equal(hio.read_image(p), rgb.astype(np.float64))


def test_ascii_pnm_and_comments(tmp_path):
    p = tmp_path / "c.pgm"
    p.write_text("P2\n# a comment\n3 2\n# another\n255\n0 1 2\n3 4 255\n")
    assert np.array_equal(hio.read_pnm(str(p)), np.array([[0, 1, 2], [3, 4, 255]], dtype=np.float64))


def test_png_filters(tmp_path):
    """Rows written with the Sub, Up, Average and Paeth filters decode to the image."""
    import struct
    import zlib
    img = np.random.default_rng(5).integers(0, 256, size=(6, 9)).astype(np.int64)
    H, W = img.shape
    raw = b""
    prev = np.zeros(W, dtype=np.int64)
    for y in range(H):
        ftype = y % 5
        row = img[y]
        enc = np.zeros(W, dtype=np.int64)
        for x in range(W):
            a = row[x - 1] if x else 0
            b = prev[x]
            c = prev[x - 1] if x else 0
            pred = [0, a, b, (a + b) >> 1, hio._paeth(a, b, c)][ftype]
            enc[x] = (row[x] - pred) & 255
        raw += bytes([ftype]) + enc.astype(np.uint8).tobytes()
        prev = row

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body))

    p = str(tmp_path / "f.png")
    with open(p, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, 8, 0, 0, 0, 0))
                + chunk(b"IDAT", zlib.compress(raw)) + chunk(b"IEND", b""))
    assert np.array_equal(hio.read_png(p), img.astype(np.float64))


def test_conversions(tmp_path, img):
    p = str(tmp_path / "d.pgm")
    hio.write_image(p, img)
    pdf, W, H, s = hio.load_img_to_pdf(p)
    ref = img.reshape(-1).astype(np.float64) + 1e-12
    assert (W, H) == (53, 37) and abs(s - ref.sum()) < 1e-6
    assert np.allclose(pdf, ref / ref.sum(), rtol=0, atol=1e-15)
    g, *_ = hio.load_img_to_pdf_gamma_correction(p, 2.0, True)
    r2 = ((255.0 - img.reshape(-1)) / 255.0) ** 2 + 1e-12
    assert np.allclose(g, r2 / r2.sum(), rtol=1e-13, atol=0)
    rgb = np.stack([img, img[::-1], 255 - img], axis=-1)
    q = str(tmp_path / "e.ppm")
    hio.write_image(q, rgb)
    lum, *_ = hio.load_rgb_img_to_pdf_grayscale_luma(q)
    r3 = (0.216 * rgb[..., 0] + 0.7152 * rgb[..., 1] + 0.0722 * rgb[..., 2]).reshape(-1) + 1e-12
    assert np.allclose(lum, r3 / r3.sum(), rtol=1e-13, atol=0)


def test_quantile_matches_reference_rule():
    d = np.array([5.0, 1.0, 4.0, 2.0, 3.0])
    # center = -0.5 + 5 p: p = 0.5 -> 2.0 -> the middle order statistic
    assert hio.quantile(d, [0.5]) == [3.0]
    # p = 0.95 -> center 4.25: clamped to the largest
    assert hio.quantile(d, [0.95])[0] == 5.0
    # p = 0.3 -> center 1.0 -> second smallest
    assert hio.quantile(d, [0.3])[0] == 2.0
    with pytest.raises(ValueError):
        hio.quantile([1.0, 2.0], [0.5])


def test_exporters(tmp_path):
    rng = np.random.default_rng(6)
    hists = [rng.random(12 * 10) for _ in range(2)]
    names = ["h0", "h1"]
    d = str(tmp_path)
    assert hio.ExportHistogramToCSV(d, digits=17).exportHistogramsBatch(hists, names) == 0
    # the reference's reader takes the last value twice when the file ends with a newline
    h = np.append(hists[0], hists[0][-1])
    assert np.array_equal(hio.load_csv_to_pdf(os.path.join(d, "h0.csv"))[0], h / h.sum())
    assert hio.ExportHistogramToCSV(d).exportHistogram(np.array([1.0 / 3, 12345678.0]), "g") == 0
    assert open(os.path.join(d, "g.csv")).read() == "0.333333\n1.23457e+07\n"
    assert hio.ExportHistogramToRAW(d).exportHistogramsBatch(hists, names) == 0
    assert np.array_equal(hio.load_raw(os.path.join(d, "h1.raw")), hists[1])
    assert hio.ExportHistogramToImage(12, 10, d).exportHistogram(hists[0], "i0") == 0
    im = hio.read_image(os.path.join(d, "i0.png"))
    q = hio.quantile(hists[0], [0.95])[0]
    assert im.shape == (10, 12, 3) and (im == im[:, :, :1]).all()  # grey in three channels
    assert np.array_equal(im[:, :, 0], np.clip(hists[0].reshape(10, 12) * 255 * 0.95 / q, 0, 255).astype(np.uint8))
    ex = hio.ExportHistogramToImageWithScaling(12, 10, [2.0, 3.0], d, alpha=1.0, complement=True)
    assert ex.exportHistogramsBatch(hists, names) == 0
    im1 = hio.read_image(os.path.join(d, "h1.png"))[:, :, 0]
    assert np.array_equal(im1, np.clip(255 - hists[1].reshape(10, 12) * 3.0 * 255, 0, 255).astype(np.uint8))
    assert hio.ExportHistogramToCSV(d).exportHistogramsBatch(hists, ["x"]) == -1


# ---- against the reference's own loaders and exporters (golden histio_ref) ----------
def _ref_fixture():
    from conftest import golden
    (_, f), = golden("histio_ref")
    return f


def _write(tmp_path, name, arr):
    p = str(tmp_path / name)
    open(p, "wb").write(bytes(arr))
    return p


def test_loaders_match_reference_cimg(tmp_path):
    """load_img_to_pdf / _grayscale_luma / _gamma_correction / load_csv_to_pdf on the
    PGM / PPM / CSV files the reference read through CImg (cpp/histogramIO.h:243-337)."""
    from wassersteindictionarylearning_b200 import histio
    f = _ref_fixture()
    W, H = int(f["W"]), int(f["H"])
    pgm = _write(tmp_path, "a.pgm", f["pgm"])
    ppm = _write(tmp_path, "a.ppm", f["ppm"])
    csv = _write(tmp_path, "a.csv", f["csv"])
    pdf, w, h, s = histio.load_img_to_pdf(pgm)
    assert (w, h) == (W, H)
    assert np.allclose(pdf, f["pdf_gray"], rtol=1e-14, atol=0) and abs(s - float(f["sum_gray"])) < 1e-9
    pdf, _, _, s = histio.load_img_to_pdf(ppm)  # first channel of an RGB file
    assert np.allclose(pdf, f["pdf_ppm_first"], rtol=1e-14, atol=0)
    pdf, _, _, s = histio.load_rgb_img_to_pdf_grayscale_luma(ppm)
    assert np.allclose(pdf, f["pdf_luma"], rtol=1e-14, atol=0) and abs(s / float(f["sum_luma"]) - 1) < 1e-14
    for alpha, comp in ((0.5, 0), (2.2, 1)):
        pdf, _, _, s = histio.load_img_to_pdf_gamma_correction(pgm, alpha, bool(comp))
        assert np.allclose(pdf, f[f"pdf_gamma_{alpha}_{comp}"], rtol=1e-13, atol=0)
        assert abs(s / float(f[f"sum_gamma_{alpha}_{comp}"]) - 1) < 1e-13
    pdf, s = histio.load_csv_to_pdf(csv)
    assert np.allclose(pdf, f["pdf_csv"], rtol=1e-15, atol=0)


def test_exporters_write_the_reference_bytes(tmp_path):
    """save_pdf / save_pdf_gamma_correction write the same PNM file as the reference
    (three replicated channels, truncation to unsigned char, cpp/histogramIO.h:339-371)."""
    from wassersteindictionarylearning_b200 import histio
    f = _ref_fixture()
    W, H = int(f["W"]), int(f["H"])
    val = f["pdf_gray"]
    p1, p2 = str(tmp_path / "o1.ppm"), str(tmp_path / "o2.ppm")
    histio.save_pdf(p1, W, H, val, float(f["save_pdf_scaling"]))
    assert open(p1, "rb").read() == bytes(f["save_pdf_bytes"])
    histio.save_pdf_gamma_correction(p2, W, H, val, 2.2, True, float(f["save_gamma_scaling"]))
    assert open(p2, "rb").read() == bytes(f["save_gamma_bytes"])


def test_quantile_matches_reference():
    from wassersteindictionarylearning_b200 import histio
    f = _ref_fixture()
    q = histio.quantile(f["quantile_data"], list(f["quantile_probs"]))
    assert np.allclose(q, f["quantile"], rtol=1e-15, atol=0)
