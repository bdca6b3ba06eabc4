"""Histogram I/O around the hot path: images and files to normalised
histograms and back, without ImageMagick.

The reference reads and writes images through CImg, which shells out to
ImageMagick / GraphicsMagick for PNG (cpp/histogramIO.h:243-371).  This module
restates those conversions on numpy arrays and reads / writes the formats
itself: binary and ASCII PNM (P2, P3, P5, P6), 8-bit PNG (grey, grey+alpha,
RGB, RGBA; decoded with zlib), one-column CSV and raw float64.

Conversions (same arithmetic as the reference):
  load_img_to_pdf              first channel + 1e-12, normalised      (:243-261)
  load_rgb_img_to_pdf_grayscale_luma  0.216 R + 0.7152 G + 0.0722 B + 1e-12 (:269-285)
  load_img_to_pdf_gamma_correction    ((255-v)/255)^a or (v/255)^a + 1e-12 (:287-310)
  load_csv_to_pdf              one value per line, normalised          (:314-337)
  save_pdf                     clamp(v * scaling, 0, 255), grey        (:339-351)
  save_pdf_gamma_correction    255 (v s)^(1/a), or its complement      (:353-369)
  quantile                     linear interpolation between order statistics (:379-405)
and the exporters of cpp/histogramIO.h:41-235 (CSV, image with the 0.95
quantile scaling, RAW float64), per histogram or in batches.
"""
from __future__ import annotations

import os
import struct
import zlib

import numpy as np

# ---------------------------------------------------------------- file formats ------


def _pnm_tokens(data: bytes, count: int, pos: int):
    """`count` whitespace-separated header tokens from pos (comments skipped)."""
    out = []
    n = len(data)
    while len(out) < count:
        while pos < n and data[pos:pos + 1].isspace():
            pos += 1
        if pos < n and data[pos:pos + 1] == b"#":
            while pos < n and data[pos:pos + 1] not in (b"\n", b"\r"):
                pos += 1
            continue
        start = pos
        while pos < n and not data[pos:pos + 1].isspace() and data[pos:pos + 1] != b"#":
            pos += 1
        if start == pos:
            raise ValueError("truncated PNM header")
        out.append(data[start:pos])
    return out, pos


def read_pnm(path: str) -> np.ndarray:
    """PNM image as an (H, W) or (H, W, 3) float64 array of sample values."""
    data = open(path, "rb").read()
    magic = data[:2]
    if magic not in (b"P2", b"P3", b"P5", b"P6"):
        raise ValueError(f"{path}: not a PGM/PPM file")
    (w, h, mx), pos = _pnm_tokens(data, 3, 2)
    W, H, maxval = int(w), int(h), int(mx)
    ch = 3 if magic in (b"P3", b"P6") else 1
    if magic in (b"P2", b"P3"):
        vals = np.array(data[pos:].split()[: W * H * ch], dtype=np.float64)
    else:
        pos += 1  # the single whitespace after maxval
        dt = np.dtype(">u2") if maxval > 255 else np.dtype(np.uint8)
        vals = np.frombuffer(data, dtype=dt, count=W * H * ch, offset=pos).astype(np.float64)
    if vals.size != W * H * ch:
        raise ValueError(f"{path}: truncated PNM data")
    return vals.reshape(H, W, ch) if ch == 3 else vals.reshape(H, W)


def write_pnm(path: str, img: np.ndarray) -> None:
    """(H, W) grey -> binary PGM, (H, W, 3) -> binary PPM, 8-bit samples."""
    a = np.asarray(img)
    magic = b"P6" if a.ndim == 3 else b"P5"
    H, W = a.shape[:2]
    with open(path, "wb") as f:
        f.write(magic + f"\n{W} {H}\n255\n".encode())
        f.write(np.ascontiguousarray(a, dtype=np.uint8).tobytes())


def _paeth(a: int, b: int, c: int) -> int:
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    if pa <= pb and pa <= pc:
        return a
    return b if pb <= pc else c


def read_png(path: str) -> np.ndarray:
    """8-bit, non-interlaced PNG (grey, grey+alpha, RGB, RGBA) as an (H, W)
    or (H, W, C) float64 array of sample values."""
    data = open(path, "rb").read()
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        raise ValueError(f"{path}: not a PNG file")
    pos, idat, ihdr = 8, [], None
    while pos < len(data):
        (length,) = struct.unpack(">I", data[pos:pos + 4])
        kind = data[pos + 4:pos + 8]
        body = data[pos + 8:pos + 8 + length]
        pos += 12 + length
        if kind == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat.append(body)
        elif kind == b"IEND":
            break
    if ihdr is None:
        raise ValueError(f"{path}: no IHDR chunk")
    W, H, depth, ctype, _, _, interlace = ihdr
    channels = {0: 1, 2: 3, 4: 2, 6: 4}.get(ctype)
    if depth != 8 or channels is None or interlace != 0:
        raise ValueError(f"{path}: only 8-bit non-interlaced grey/RGB(A) PNG is supported")
    raw = zlib.decompress(b"".join(idat))
    stride = W * channels
    out = np.zeros((H, stride), dtype=np.uint8)
    prev = np.zeros(stride, dtype=np.int64)
    for y in range(H):
        ftype = raw[y * (stride + 1)]
        line = np.frombuffer(raw, dtype=np.uint8, count=stride, offset=y * (stride + 1) + 1).astype(np.int64)
        if ftype == 0:
            cur = line
        elif ftype == 2:
            cur = (line + prev) & 255
        else:  # Sub, Average, Paeth depend on the reconstructed left neighbour
            cur = np.zeros(stride, dtype=np.int64)
            for x in range(stride):
                left = cur[x - channels] if x >= channels else 0
                up = prev[x]
                if ftype == 1:
                    pred = left
                elif ftype == 3:
                    pred = (left + up) >> 1
                elif ftype == 4:
                    pred = _paeth(left, up, prev[x - channels] if x >= channels else 0)
                else:
                    raise ValueError(f"{path}: bad PNG filter {ftype}")
                cur[x] = (line[x] + pred) & 255
        out[y] = cur
        prev = cur
    img = out.reshape(H, W, channels).astype(np.float64)
    return img[:, :, 0] if channels == 1 else img


def write_png(path: str, img: np.ndarray) -> None:
    """(H, W) grey or (H, W, 3) RGB 8-bit PNG (filter None, zlib level 6)."""
    a = np.ascontiguousarray(np.asarray(img), dtype=np.uint8)
    H, W = a.shape[:2]
    ctype = 2 if a.ndim == 3 else 0
    rows = a.reshape(H, -1)
    raw = b"".join(b"\x00" + rows[y].tobytes() for y in range(H))

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, 8, ctype, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def read_image(path: str) -> np.ndarray:
    """PNG or PNM by content."""
    head = open(path, "rb").read(8)
    return read_png(path) if head.startswith(b"\x89PNG") else read_pnm(path)


def write_image(path: str, img: np.ndarray) -> None:
    """PNG for a .png name, PNM otherwise."""
    (write_png if path.lower().endswith(".png") else write_pnm)(path, img)


def _planes(img: np.ndarray) -> np.ndarray:
    return img if img.ndim == 3 else img[:, :, None]

# ---------------------------------------------------------------- conversions -------


def load_img_to_pdf(path: str):
    """(pdf [W*H], W, H, sum): the first channel + 1e-12, normalised to 1 (the
    reference reads CImg's data(), whose first plane is the first channel)."""
    img = _planes(read_image(path))
    H, W = img.shape[:2]
    v = img[:, :, 0].reshape(-1) + 1e-12
    s = float(v.sum())
    return v / s, W, H, s


def load_rgb_img_to_pdf_grayscale_luma(path: str):
    img = _planes(read_image(path))
    if img.shape[2] < 3:
        raise ValueError(f"{path}: not an RGB image")
    H, W = img.shape[:2]
    v = (0.216 * img[:, :, 0] + 0.7152 * img[:, :, 1] + 0.0722 * img[:, :, 2]).reshape(-1) + 1e-12
    s = float(v.sum())
    return v / s, W, H, s


def load_img_to_pdf_gamma_correction(path: str, alpha: float, complement: bool):
    img = _planes(read_image(path))
    H, W = img.shape[:2]
    c = img[:, :, 0].reshape(-1)
    v = (((255.0 - c) / 255.0) if complement else (c / 255.0)) ** alpha + 1e-12
    s = float(v.sum())
    return v / s, W, H, s


def load_csv_to_pdf(path: str):
    """(pdf, sum) as the reference's loop `while (ifs.good()) { ifs >> v; sum += v;
    result.push_back(v); }` (cpp/histogramIO.h:314-337) reads it: when the file
    ends with whitespace the extraction after the last value fails before
    touching v, so the last value is appended (and summed) a second time; a
    token that is not a number stores 0 and ends the loop."""
    text = open(path).read()
    vals = []
    failed = False
    for tok in text.split():
        try:
            v = float(tok)
            if not np.isfinite(v) and tok.lower().lstrip("+-") in ("nan", "inf", "infinity"):
                raise ValueError(tok)  # iostream does not parse these words
        except ValueError:
            failed = True
            break
        vals.append(v)
    if failed:
        vals.append(0.0)
    elif not vals:
        raise ValueError(f"{path}: no values (the reference reads an uninitialised value here)")
    elif text[-1:].isspace():
        vals.append(vals[-1])
    v = np.array(vals, dtype=np.float64)
    s = float(v.sum())
    return v / s, s


def load_raw(path: str) -> np.ndarray:
    return np.fromfile(path, dtype=np.float64)


def _to_u8(v: np.ndarray) -> np.ndarray:
    # the reference stores min(255, max(0, x)) into unsigned char (truncation)
    return np.clip(v, 0.0, 255.0).astype(np.uint8)


def _rgb(gray: np.ndarray) -> np.ndarray:
    # the reference replicates the grey plane into three channels before saving
    # (cpp/histogramIO.h:341-347), so its files are RGB
    return np.repeat(gray[:, :, None], 3, axis=2)


def save_pdf(path: str, W: int, H: int, val, scaling: float) -> None:
    write_image(path, _rgb(_to_u8(np.asarray(val, dtype=np.float64).reshape(H, W) * scaling)))


def save_pdf_gamma_correction(path: str, W: int, H: int, val, alpha: float, complement: bool,
                              scaling: float) -> None:
    g = np.power(np.asarray(val, dtype=np.float64).reshape(H, W) * scaling, 1.0 / alpha) * 255.0
    write_image(path, _rgb(_to_u8(255.0 - g if complement else g)))


def quantile(data, probs):
    """Linear-interpolation quantiles as cpp/histogramIO.h:379-405."""
    d = np.sort(np.asarray(data, dtype=np.float64).reshape(-1))
    if d.size <= 2 or len(probs) == 0:
        raise ValueError("Invalid input")
    out = []
    for p in probs:
        center = (1 - p) * (-0.5) + p * (d.size - 0.5)
        left = max(int(np.floor(center)), 0)
        right = min(int(np.ceil(center)), d.size - 1)
        t = center - left
        out.append((1 - t) * d[left] + t * d[right])
    return out

# ---------------------------------------------------------------- exporters ---------


class ExportHistogramToCSV:
    """One value per line, written as the reference's ostream does by default
    (6 significant digits, %g); `digits=17` writes them losslessly."""

    def __init__(self, folder: str = "outputFiles", digits: int = 6):
        self.folder = folder
        self.digits = digits

    def exportHistogram(self, results, name: str) -> int:
        fmt = f"%.{self.digits}g\n"
        try:
            with open(os.path.join(self.folder, name + ".csv"), "w") as f:
                for v in np.asarray(results, dtype=np.float64).reshape(-1):
                    f.write(fmt % float(v))
        except OSError:
            return -1
        return 0

    def exportHistogramsBatch(self, results, names) -> int:
        if len(results) != len(names):
            return -1
        return 0 if all(self.exportHistogram(r, n) == 0 for r, n in zip(results, names)) else -1


class ExportHistogramToImage(ExportHistogramToCSV):
    """The reference's PNG exporter (cpp/histogramIO.h:101-137): grey image
    scaled so that the 0.95 quantile maps to 0.95 * 255."""

    def __init__(self, width: int, height: int, folder: str = "outputFiles", ext: str = ".png"):
        super().__init__(folder)
        self.W, self.H, self.ext = width, height, ext

    def exportHistogram(self, results, name: str) -> int:
        r = np.asarray(results, dtype=np.float64).reshape(-1)
        if r.size != self.W * self.H:
            return -1
        q = quantile(r, [0.95])[0]
        try:
            save_pdf(os.path.join(self.folder, name + self.ext), self.W, self.H, r, 255.0 * 0.95 / q)
        except OSError:
            return -1
        return 0


class ExportHistogramToRAW(ExportHistogramToCSV):
    def exportHistogram(self, results, name: str) -> int:
        try:
            np.asarray(results, dtype=np.float64).reshape(-1).tofile(os.path.join(self.folder, name + ".raw"))
        except OSError:
            return -1
        return 0


class ExportHistogramToImageWithScaling(ExportHistogramToCSV):
    """The reference's gamma-corrected exporter with stored scalings
    (cpp/histogramIO.h:140-199): exportHistogram uses the 0.95 quantile,
    exportHistogramsBatch applies scalings[i] to result i (the scalings are
    those returned when the inputs were loaded, so each reconstruction is
    written at its input's scale)."""

    def __init__(self, width: int, height: int, scalings, folder: str = "outputFiles",
                 alpha: float = 1.0, complement: bool = False, ext: str = ".png"):
        super().__init__(folder)
        self.W, self.H, self.scalings = width, height, list(scalings)
        self.alpha, self.complement, self.ext = alpha, complement, ext

    def _save(self, r, name, scaling) -> int:
        try:
            save_pdf_gamma_correction(os.path.join(self.folder, name + self.ext), self.W, self.H, r,
                                      self.alpha, self.complement, scaling)
        except OSError:
            return -1
        return 0

    def exportHistogram(self, results, name: str) -> int:
        r = np.asarray(results, dtype=np.float64).reshape(-1)
        if r.size != self.W * self.H:
            return -1
        return self._save(r, name, 0.95 / quantile(r, [0.95])[0])

    def exportHistogramsBatch(self, results, names) -> int:
        if len(results) != len(names):
            return -1
        ok = True
        for i, (r, n) in enumerate(zip(results, names)):
            if i >= len(self.scalings):
                ok = False
                continue
            ok = self._save(np.asarray(r, dtype=np.float64).reshape(-1), n, self.scalings[i]) == 0 and ok
        return 0 if ok else -1
