"""The asset path: scene files, OBJ/MTL meshes and textures, loaded as the reference's
frontend loads them (src/imbatracer/frontend/build_scene.cpp, src/imbatracer/loaders/).

    desc = load_scene_file("cornell/cornell_org.scene", width=512, height=512)
    gs = GpuScene(desc)                         # then PathTracer / VcmIntegrator / Server

A `.scene` file gives the camera (pos, dir, up), meshes (OBJ files, each with an optional
`accel` cache file), instances (mesh index, pos / scale / rot), directional, point and spot
lights (parse_scene_file, build_scene.cpp:315-546). Each OBJ file becomes one mesh with
vertices deduplicated per object, polygons fanned into triangles and one material per
emissive face, whose triangle becomes an area light (create_mesh, :184-304); MTL materials
map to the reference's material classes (convert_materials, :55-182): illum 5 mirror,
illum 7 glass, a non-zero Ks glossy, otherwise diffuse, with diffuse textures (map_Kd),
bump maps (map_bump / bump) and opacity masks (map_d). Arithmetic that decides results
(instance matrices, normals, light vertices) is done in single precision in the
reference's order of operations, so the arrays equal the reference's.

An `env <file.hdr> <intensity>` command gives an image environment light (load_hdr.cpp;
EnvMap, light.h:361-544); it is light 0 here, so a scene listing other lights before it
samples them in another order than the reference (same estimate, other random numbers).
Emissive materials whose base is not diffuse become emissive diffuse.
"""
from __future__ import annotations

import math
import os
import struct
import zlib
from dataclasses import dataclass, field

import numpy as np

from . import native as N
from . import scenegen as G
from .scene import Instance, Mesh

f32 = np.float32
PI_F = f32(3.14159265359)        # imba::pi (common.h)


# ---------------------------------------------------------------------------------------
# Images: load_png.cpp, load_tga.cpp, loaders.h load_image (PNG first, then TGA)
# ---------------------------------------------------------------------------------------
def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    if pa <= pb and pa <= pc:
        return a
    return b if pb <= pc else c


def _unfilter(raw: bytes, width: int, height: int, bpp: int, row_bytes: int) -> np.ndarray:
    out = np.zeros((height, row_bytes), np.uint8)
    prev = np.zeros(row_bytes, np.int32)
    pos = 0
    for y in range(height):
        ftype = raw[pos]
        line = np.frombuffer(raw, np.uint8, row_bytes, pos + 1).astype(np.int32)
        pos += 1 + row_bytes
        if ftype == 0:
            cur = line
        elif ftype == 1:     # Sub: cumulative per byte lane
            cur = line.copy()
            for k in range(bpp, row_bytes):
                cur[k] = (cur[k] + cur[k - bpp]) & 0xFF
        elif ftype == 2:     # Up
            cur = (line + prev) & 0xFF
        elif ftype == 3:     # Average
            cur = line.copy()
            for k in range(row_bytes):
                left = cur[k - bpp] if k >= bpp else 0
                cur[k] = (cur[k] + ((left + prev[k]) >> 1)) & 0xFF
        elif ftype == 4:     # Paeth
            cur = line.copy()
            for k in range(row_bytes):
                left = int(cur[k - bpp]) if k >= bpp else 0
                upleft = int(prev[k - bpp]) if k >= bpp else 0
                cur[k] = (cur[k] + _paeth(left, int(prev[k]), upleft)) & 0xFF
        else:
            raise ValueError(f"png: bad filter type {ftype}")
        out[y] = cur
        prev = cur
    return out


def load_png(path: str) -> np.ndarray | None:
    """(height, width, 4) float32 in [0, 1] (bytes / 255, no colour-space conversion), or
    None when the file is not a PNG. Palette and grey images are expanded to RGB, 16-bit
    channels cut to their high byte, a tRNS chunk becomes alpha, else alpha is 1
    (load_png.cpp:14-88). Interlaced images are not supported."""
    try:
        data = open(path, "rb").read()
    except OSError:
        return None
    if data[:8] != b"\x89PNG\r\n\x1a\n":
        return None
    pos, idat, plte, trns, hdr = 8, [], None, None, None
    while pos + 8 <= len(data):
        length, ctype = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + length]
        pos += 12 + length
        if ctype == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif ctype == b"PLTE":
            plte = np.frombuffer(body, np.uint8).reshape(-1, 3)
        elif ctype == b"tRNS":
            trns = body
        elif ctype == b"IDAT":
            idat.append(body)
        elif ctype == b"IEND":
            break
    if hdr is None:
        return None
    w, h, depth, ctype, _, _, interlace = hdr
    if interlace != 0:
        raise ValueError(f"png: interlaced images are not supported ({path})")
    channels = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
    if ctype == 3:
        if depth not in (1, 2, 4, 8):
            raise ValueError("png: bad palette depth")
    elif depth not in (8, 16):
        raise ValueError(f"png: bit depth {depth} is not supported ({path})")
    bits = channels * depth
    row_bytes = (w * bits + 7) // 8
    bpp = max(1, bits // 8)
    rows = _unfilter(zlib.decompress(b"".join(idat)), w, h, bpp, row_bytes)
    if ctype == 3:
        if depth < 8:
            per = 8 // depth
            shifts = (8 - depth) - depth * (np.arange(w) % per)
            idx = (rows[:, np.arange(w) // per] >> shifts) & ((1 << depth) - 1)
        else:
            idx = rows[:, :w]
        rgb = plte[idx]
        alpha = np.full((h, w), 255, np.uint8)
        if trns is not None:
            table = np.full(256, 255, np.uint8)
            table[:len(trns)] = np.frombuffer(trns, np.uint8)
            alpha = table[idx]
        px = np.concatenate([rgb, alpha[..., None]], -1)
    else:
        v = rows.reshape(h, -1)
        if depth == 16:
            v = v.reshape(h, w * channels, 2)[..., 0]      # png_set_strip_16: the high byte
        v = v.reshape(h, w, channels)
        if ctype in (0, 4):
            grey = v[..., :1]
            rgb = np.repeat(grey, 3, -1)
            alpha = v[..., 1:2] if ctype == 4 else None
        else:
            rgb = v[..., :3]
            alpha = v[..., 3:4] if ctype == 6 else None
        if alpha is None:
            alpha = np.full((h, w, 1), 255, np.uint8)
            if trns is not None and ctype in (0, 2):
                key = np.frombuffer(trns, ">u2")
                key = (key >> 8).astype(np.uint8) if depth == 16 else key.astype(np.uint8)
                match = np.all(rgb == (key[0] if ctype == 0 else key[:3]), -1)
                alpha = np.where(match, 0, 255).astype(np.uint8)[..., None]
        px = np.concatenate([rgb, alpha], -1)
    return (px.astype(np.float32) / f32(255.0)).astype(np.float32)


def load_tga(path: str) -> np.ndarray | None:
    """Uncompressed (type 2, stored bottom-up) and RLE (type 10, rows kept in file order, as
    the reference does) 24/32-bit TGA files (load_tga.cpp:119-149)."""
    try:
        data = open(path, "rb").read()
    except OSError:
        return None
    if len(data) < 18:
        return None
    raw_sig = bytes([0, 0, 2] + [0] * 9)
    comp_sig = bytes([0, 0, 10] + [0] * 9)
    kind = "raw" if data[:12] == raw_sig else "rle" if data[:12] == comp_sig else None
    if kind is None:
        return None
    w, h, bpp, _ = struct.unpack("<HHBB", data[12:18])
    if w <= 0 or h <= 0 or bpp not in (24, 32):
        return None
    nb = bpp // 8
    img = np.zeros((h * w, 4), np.float32)
    body = np.frombuffer(data, np.uint8, offset=18)
    inv = f32(255.0)

    def put(dst, pix):
        img[dst, 2] = pix[:, 0] / inv
        img[dst, 1] = pix[:, 1] / inv
        img[dst, 0] = pix[:, 2] / inv
        img[dst, 3] = pix[:, 3] / inv if nb == 4 else f32(1.0)

    if kind == "raw":
        need = w * h * nb
        pix = body[:need].reshape(h, w, nb)
        if len(pix.reshape(-1)) < need:
            return None
        for y in range(h):
            put(np.arange((h - 1 - y) * w, (h - y) * w), pix[y])
    else:
        cur, p, n = 0, 0, w * h
        while cur < n and p < len(body):
            chunk = int(body[p]); p += 1
            if chunk < 128:
                chunk += 1
                pix = body[p:p + chunk * nb].reshape(-1, nb)
                p += chunk * nb
                chunk = min(chunk, n - cur)
                put(np.arange(cur, cur + chunk), pix[:chunk])
            else:
                chunk -= 127
                one = np.array(list(body[p:p + nb]) + ([255] if nb == 3 else []), np.uint8)
                p += nb
                chunk = min(chunk, n - cur)
                img[cur:cur + chunk] = np.array([one[2], one[1], one[0], one[3]], np.float32) / inv
            cur += chunk
    return img.reshape(h, w, 4)


def load_hdr(path: str) -> np.ndarray:
    """Radiance RGBE images with run-length encoded scanlines (load_hdr.cpp:174-229): header
    lines up to an empty line, a "-Y height +X width" resolution line, one scanline per row;
    texel = ((byte + 0.5) * 2^(e - 136)) per channel, alpha 0. Scanlines in the older flat or
    RLE formats are refused: the reference's decoder does not store their pixels."""
    data = open(path, "rb").read()
    pos = data.index(b"\n") + 1                    # the signature line (not checked)
    while True:
        end = data.index(b"\n", pos)
        line = data[pos:end]
        pos = end + 1
        if line == b"":
            break
    end = data.index(b"\n", pos)
    res = data[pos:end].split()
    pos = end + 1
    if len(res) != 4 or res[0] != b"-Y" or res[2] != b"+X":
        raise ValueError(f"hdr: unsupported axis configuration in {path}")
    h, w = int(res[1]), int(res[3])
    img = np.zeros((h, w, 4), np.float32)
    buf = np.frombuffer(data, np.uint8)
    for y in range(h):
        if pos + 4 > len(buf):
            raise ValueError(f"hdr: unexpected end of file in {path}")
        r, g, b, e = (int(v) for v in buf[pos:pos + 4])
        pos += 4
        if not (r == 2 and g == 2 and not (b & 128)):
            raise ValueError(f"hdr: only adaptive run-length scanlines are supported ({path})")
        if ((b << 8) | e) != w:
            raise ValueError(f"hdr: scanline length mismatch in {path}")
        px = np.zeros((w, 4), np.uint8)
        for comp in range(4):
            i = 0
            while i < w:
                code = int(buf[pos]); pos += 1
                if code > 128:
                    code &= 127
                    if i + code > w:
                        raise ValueError("hdr: overrun in a scanline run")
                    px[i:i + code, comp] = buf[pos]; pos += 1
                    i += code
                else:
                    if code == 0 or i + code > w:
                        raise ValueError("hdr: bad scanline dump")
                    px[i:i + code, comp] = buf[pos:pos + code]; pos += code
                    i += code
        scale = np.ldexp(1.0, px[:, 3].astype(np.int64) - 136)
        for c in range(3):
            img[y, :, c] = ((px[:, c].astype(np.float64) + 0.5) * scale).astype(np.float32)
    return img


def load_image(path: str) -> np.ndarray | None:
    img = load_png(path)
    return img if img is not None else load_tga(path)


# ---------------------------------------------------------------------------------------
# OBJ / MTL (load_obj.cpp)
# ---------------------------------------------------------------------------------------
@dataclass
class ObjMaterial:
    ka: tuple = (0.0, 0.0, 0.0)
    kd: tuple = (0.0, 0.0, 0.0)
    ks: tuple = (0.0, 0.0, 0.0)
    ke: tuple = (0.0, 0.0, 0.0)
    ns: float = 0.0
    ni: float = 0.0
    tf: tuple = (0.0, 0.0, 0.0)
    tr: float = 0.0
    d: float = 0.0
    illum: int = 0
    map_ka: str = ""
    map_kd: str = ""
    map_ks: str = ""
    map_ke: str = ""
    map_bump: str = ""
    map_d: str = ""


@dataclass
class ObjFile:
    objects: list = field(default_factory=lambda: [[[]]])     # objects -> groups -> faces
    vertices: list = field(default_factory=lambda: [(0.0, 0.0, 0.0)])
    normals: list = field(default_factory=lambda: [(0.0, 0.0, 0.0)])
    texcoords: list = field(default_factory=lambda: [(0.0, 0.0)])
    materials: list = field(default_factory=lambda: [""])
    mtl_libs: list = field(default_factory=list)


def _strtof(s: str, pos: int) -> tuple[float, int]:
    """std::strtof: skips spaces, parses the longest number prefix; 0 and no advance when
    there is none."""
    n = len(s)
    i = pos
    while i < n and s[i].isspace():
        i += 1
    j = i
    if j < n and s[j] in "+-":
        j += 1
    digits = 0
    while j < n and s[j].isdigit():
        j += 1; digits += 1
    if j < n and s[j] == ".":
        j += 1
        while j < n and s[j].isdigit():
            j += 1; digits += 1
    if digits == 0:
        low = s[i:i + 9].lower().lstrip("+-")
        for word in ("infinity", "inf", "nan"):
            if low.startswith(word):
                j = i + (len(s[i:]) - len(s[i:].lstrip("+-"))) + len(word)
                return float(np.float32(s[i:j])), j
        return 0.0, pos
    if j < n and s[j] in "eE":
        k = j + 1
        if k < n and s[k] in "+-":
            k += 1
        if k < n and s[k].isdigit():
            while k < n and s[k].isdigit():
                k += 1
            j = k
    return float(np.float32(s[i:j])), j


def _strtol(s: str, pos: int) -> tuple[int, int]:
    n = len(s)
    i = pos
    while i < n and s[i].isspace():
        i += 1
    j = i
    if j < n and s[j] in "+-":
        j += 1
    k = j
    while k < n and s[k].isdigit():
        k += 1
    if k == j:
        return 0, pos
    return int(s[i:k]), k


def _read_index(s: str, pos: int):
    """read_index (load_obj.cpp:43-77): v[/[t][/n]], negative indices allowed."""
    n = len(s)
    while pos < n and s[pos].isspace():
        pos += 1
    if pos >= n or not (s[pos].isdigit() or s[pos] == "-"):
        return None, pos
    v, pos = _strtol(s, pos)
    t = nn = 0
    while pos < n and s[pos].isspace():
        pos += 1
    if pos < n and s[pos] == "/":
        pos += 1
        if pos < n and s[pos] != "/":
            t, pos = _strtol(s, pos)
        while pos < n and s[pos].isspace():
            pos += 1
        if pos < n and s[pos] == "/":
            pos += 1
            nn, pos = _strtol(s, pos)
    return (v, t, nn), pos


def parse_obj(path: str) -> ObjFile:
    """parse_obj (load_obj.cpp:79-218). Raises ValueError when the reference's loader
    reports errors (it then refuses the file)."""
    f = ObjFile()
    cur_obj, cur_grp, cur_mtl, errors = 0, 0, 0, 0
    with open(path, "r", errors="replace") as fh:
        for line in fh:
            s = line.strip()
            if not s or s[0] == "#":
                continue
            if s[0] == "v":
                c = s[1] if len(s) > 1 else ""
                if c in (" ", "\t"):
                    x, p = _strtof(s, 1); y, p = _strtof(s, p); z, p = _strtof(s, p)
                    f.vertices.append((x, y, z))
                elif c == "n":
                    x, p = _strtof(s, 2); y, p = _strtof(s, p); z, p = _strtof(s, p)
                    f.normals.append((x, y, z))
                elif c == "t":
                    x, p = _strtof(s, 2); y, p = _strtof(s, p)
                    f.texcoords.append((x, y))
                else:
                    errors += 1
            elif s[0] == "f" and len(s) > 1 and s[1].isspace():
                idx, p = [], 2
                while len(idx) < 8:
                    r, p = _read_index(s, p)
                    if r is None:
                        break
                    idx.append(r)
                if len(idx) < 3:
                    errors += 1
                    continue
                nv, nt, nn = len(f.vertices), len(f.texcoords), len(f.normals)
                idx = [(v + nv if v < 0 else v, t + nt if t < 0 else t, n + nn if n < 0 else n) for v, t, n in idx]
                if any(v <= 0 or t < 0 or n < 0 for v, t, n in idx):
                    errors += 1
                    continue
                f.objects[cur_obj][cur_grp].append((idx, cur_mtl))
            elif s[0] == "g" and len(s) > 1 and s[1].isspace():
                f.objects[cur_obj].append([])
                cur_grp += 1
            elif s[0] == "o" and len(s) > 1 and s[1].isspace():
                f.objects.append([[]])
                cur_obj += 1
                cur_grp = 0
            elif s.startswith("usemtl") and len(s) > 6 and s[6].isspace():
                name = s[6:].split()[0] if s[6:].split() else ""
                if name in f.materials:
                    cur_mtl = f.materials.index(name)
                else:
                    f.materials.append(name)
                    cur_mtl = len(f.materials) - 1
            elif s.startswith("mtllib") and len(s) > 6 and s[6].isspace():
                parts = s[6:].split()
                f.mtl_libs.append(parts[0] if parts else "")
            elif s[0] == "s" and len(s) > 1 and s[1].isspace():
                pass
            else:
                errors += 1
    if errors:
        raise ValueError(f"obj: {errors} invalid line(s) in {path}")
    return f


def parse_mtl(path: str, lib: dict) -> None:
    """parse_mtl (load_obj.cpp:220-348) into `lib` (name -> ObjMaterial)."""
    name, errors = "", 0

    def cur():
        return lib.setdefault(name, ObjMaterial())

    def vec3(s, p):
        x, p = _strtof(s, p); y, p = _strtof(s, p); z, p = _strtof(s, p)
        return (x, y, z)

    with open(path, "r", errors="replace") as fh:
        for line in fh:
            s = line.strip()
            if not s or s[0] == "#":
                continue
            if s.startswith("newmtl") and len(s) > 6 and s[6].isspace():
                parts = s[7:].split()
                name = parts[0] if parts else ""
                if name in lib:
                    errors += 1
            elif s[0] == "K" and len(s) > 2 and s[2].isspace() and s[1] in "adse":
                setattr(cur(), "k" + s[1], vec3(s, 3))
            elif s[0] == "N" and len(s) > 2 and s[2].isspace() and s[1] in "si":
                setattr(cur(), "n" + s[1], _strtof(s, 3)[0])
            elif s[0] == "T" and len(s) > 2 and s[2].isspace() and s[1] == "f":
                cur().tf = vec3(s, 3)
            elif s[0] == "T" and len(s) > 2 and s[2].isspace() and s[1] == "r":
                cur().tr = _strtof(s, 3)[0]
            elif s[0] == "d" and len(s) > 1 and s[1].isspace():
                cur().d = _strtof(s, 2)[0]
            elif s.startswith("illum") and len(s) > 5 and s[5].isspace():
                cur().illum = int(_strtof(s, 6)[0])
            elif any(s.startswith(k) and len(s) > len(k) and s[len(k)].isspace()
                     for k in ("map_Ka", "map_Kd", "map_Ks", "map_Ke", "map_bump", "map_Bump", "bump", "map_d")):
                key = s.split()[0]
                value = s[len(key) + 1:].strip()
                attr = {"map_Ka": "map_ka", "map_Kd": "map_kd", "map_Ks": "map_ks", "map_Ke": "map_ke",
                        "map_bump": "map_bump", "map_Bump": "map_bump", "bump": "map_bump", "map_d": "map_d"}[key]
                setattr(cur(), attr, value)
            else:
                errors += 1
    if errors:
        raise ValueError(f"mtl: {errors} invalid line(s) in {path}")


# ---------------------------------------------------------------------------------------
# Scene assembly (build_scene.cpp)
# ---------------------------------------------------------------------------------------
def _dot4(a, b):
    return f32(f32(f32(f32(a[0] * b[0]) + f32(a[1] * b[1])) + f32(a[2] * b[2])) + f32(a[3] * b[3]))


def _matmul4(a, b):
    bt = b.T
    out = np.zeros((4, 4), np.float32)
    for i in range(4):
        for j in range(4):
            out[i, j] = _dot4(a[i], bt[j])
    return out


def _radians(x):
    return f32(f32(f32(x) * PI_F) / f32(180.0))


def instance_matrix(pos, scale, euler_deg) -> np.ndarray:
    """translate(pos) * euler(rx, ry, rz) * scale(s) (build_scene.cpp:494; float4x4.h:48-81,
    197-199: euler = rotate_x * rotate_y * rotate_z) in single precision."""
    ex, ey, ez = (_radians(a) for a in euler_deg)
    sin = lambda a: f32(math.sin(float(a)))
    cos = lambda a: f32(math.cos(float(a)))
    rx = np.array([[1, 0, 0, 0], [0, cos(ex), sin(ex), 0], [0, -sin(ex), cos(ex), 0], [0, 0, 0, 1]], np.float32)
    ry = np.array([[cos(ey), 0, -sin(ey), 0], [0, 1, 0, 0], [sin(ey), 0, cos(ey), 0], [0, 0, 0, 1]], np.float32)
    rz = np.array([[cos(ez), sin(ez), 0, 0], [-sin(ez), cos(ez), 0, 0], [0, 0, 1, 0], [0, 0, 0, 1]], np.float32)
    t = np.array([[1, 0, 0, pos[0]], [0, 1, 0, pos[1]], [0, 0, 1, pos[2]], [0, 0, 0, 1]], np.float32)
    s = np.diag(np.array([scale[0], scale[1], scale[2], 1.0], np.float32))
    e = _matmul4(_matmul4(rx, ry), rz)
    return _matmul4(_matmul4(t, e), s)


def _normalize_rows(v: np.ndarray) -> np.ndarray:
    """a * (1 / sqrtf(dot(a, a))) per row (float3.h:114-128)."""
    d = ((v[:, 0] * v[:, 0]) + (v[:, 1] * v[:, 1])) + (v[:, 2] * v[:, 2])
    with np.errstate(divide="ignore", invalid="ignore"):
        inv = f32(1.0) / np.sqrt(d.astype(np.float32))
        return (v * inv[:, None]).astype(np.float32)


def _cross_rows(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.stack([a[:, 1] * b[:, 2] - a[:, 2] * b[:, 1],
                     a[:, 2] * b[:, 0] - a[:, 0] * b[:, 2],
                     a[:, 0] * b[:, 1] - a[:, 1] * b[:, 0]], 1).astype(np.float32)


def _face_cross(v: np.ndarray, idx: np.ndarray) -> np.ndarray:
    p0, p1, p2 = v[idx[:, 0]], v[idx[:, 1]], v[idx[:, 2]]
    return _cross_rows((p1 - p0).astype(np.float32), (p2 - p0).astype(np.float32))


def _compute_normals(v: np.ndarray, idx: np.ndarray) -> np.ndarray:
    """Mesh::compute_normals (mesh.cpp:7-27): per vertex the sum of the faces' unnormalized
    cross products in face order, normalized."""
    acc = np.zeros((len(v), 3), np.float32)
    n = _face_cross(v, idx)
    for k in range(3):
        np.add.at(acc, idx[:, k], n)
    return _normalize_rows(acc)


def _xform_point(m: np.ndarray, p) -> np.ndarray:
    q = (f32(p[0]), f32(p[1]), f32(p[2]), f32(1.0))
    return np.array([_dot4(m[r], q) for r in range(3)], np.float32)


@dataclass
class SceneFileInfo:
    mesh_files: list = field(default_factory=list)
    accel_files: list = field(default_factory=list)
    cam_pos: tuple | None = None
    cam_dir: tuple | None = None
    cam_up: tuple | None = None
    instances: list = field(default_factory=list)   # (mesh index, 4x4 matrix)
    lights: list = field(default_factory=list)      # (kind, 12 floats) in file order
    env: tuple | None = None        # (image path, intensity)


def parse_scene_file(path: str) -> SceneFileInfo:
    """parse_scene_file (build_scene.cpp:315-546): whitespace-separated commands; `#`
    comments to the end of the line; instance attributes until the first unknown or
    repeated one."""
    base = os.path.dirname(path) or "."
    text = open(path, "r", errors="replace").read()
    toks, lines = [], text.split("\n")
    for line in lines:
        for t in line.split():
            if t.startswith("#"):
                break
            toks.append(t)
    info = SceneFileInfo()
    i = 0

    def nums_after(j):
        if j >= len(toks):
            raise ValueError(f"scene: unexpected end of file in {path}")
        return float(np.float32(toks[j]))

    def nums(k):
        nonlocal i
        if i + k > len(toks):
            raise ValueError(f"scene: unexpected end of file in {path}")
        out = [float(np.float32(toks[i + j])) for j in range(k)]
        i += k
        return out

    while i < len(toks):
        cmd = toks[i]; i += 1
        if cmd == "pos":
            info.cam_pos = tuple(nums(3))
        elif cmd == "dir":
            info.cam_dir = tuple(nums(3))
        elif cmd == "up":
            info.cam_up = tuple(nums(3))
        elif cmd == "mesh":
            info.mesh_files.append(os.path.join(base, toks[i])); i += 1
            info.accel_files.append(None)
        elif cmd == "accel":
            if not info.accel_files:
                raise ValueError("scene: BVH files have to be specified after the mesh they belong to")
            info.accel_files[-1] = os.path.join(base, toks[i]); i += 1
        elif cmd == "dir_light":
            d = np.array(nums(3), np.float32)
            e = nums(3)
            n = _normalize_rows(d[None])[0]
            info.lights.append((G.DIRECTIONAL, list(map(float, n)) + [0.0] * 6 + e))
        elif cmd == "point_light":
            p = nums(3); e = nums(3)
            info.lights.append((G.POINT, p + [0.0] * 6 + e))
        elif cmd == "spot_light":
            p = nums(3)
            d = _normalize_rows(np.array(nums(3), np.float32)[None])[0]
            angle = nums(1)[0]
            e = nums(3)
            info.lights.append((G.SPOT, p + list(map(float, d)) + [float(_radians(angle)), 0.0, 0.0] + e))
        elif cmd == "instance":
            idx = int(toks[i]); i += 1
            pos, scale, rot, flags = (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (0.0, 0.0, 0.0), 0
            while flags != 7 and i < len(toks):
                c = toks[i]
                if c == "pos" and not flags & 1:
                    i += 1; pos = tuple(nums(3)); flags |= 1
                elif c == "scale" and not flags & 2:
                    i += 1; scale = tuple(nums(3)); flags |= 2
                elif c == "rot" and not flags & 4:
                    i += 1; rot = tuple(nums(3)); flags |= 4
                else:
                    break
            info.instances.append((idx, instance_matrix(pos, scale, rot)))
        elif cmd == "env":
            if info.env is not None:
                continue                            # the reference ignores further maps
            info.env = (os.path.join(base, toks[i]), nums_after(i + 1))
            i += 2
        # unknown commands are skipped, as the reference's loop does
    if info.cam_pos is None or info.cam_dir is None or info.cam_up is None:
        raise ValueError("scene: camera settings not specified")
    if not info.mesh_files:
        raise ValueError("scene: no meshes specified")
    if not info.instances:
        info.instances = [(k, np.eye(4, dtype=np.float32)) for k in range(len(info.mesh_files))]
    return info


class _Textures:
    """Scene textures, loaded once per file name (convert_materials' tex_map)."""

    def __init__(self):
        self.ids, self.images = {}, []

    def load(self, name: str) -> int:
        if name in self.ids:
            return self.ids[name]
        img = load_image(name)
        tid = -1
        if img is not None:
            tid = len(self.images)
            self.images.append(np.ascontiguousarray(img, np.float32))
        self.ids[name] = tid
        return tid


class _Masks:
    """MaskBuffer (mask.h): 4 opaque bytes, then one byte per texel (r + g + b > 0)."""

    def __init__(self):
        self.buffer = [np.ones(4, np.uint8)]
        self.size = 4
        self.descs = []

    def add(self, desc=(1, 1, 0)):
        self.descs.append(desc)

    def append(self, img: np.ndarray) -> tuple:
        h, w = img.shape[:2]
        off = self.size
        bits = ((img[..., 0] + img[..., 1] + img[..., 2]) > 0).astype(np.uint8).reshape(-1)
        self.buffer.append(bits)
        self.size += len(bits)
        self.descs.append((w, h, off))
        return w, h, off


def _convert_materials(obj_path, obj: ObjFile, lib: dict, materials: list, emissive: dict, tex: _Textures,
                       masks: _Masks, mask_ids: dict):
    base = os.path.dirname(obj_path) or "."
    materials.append(G.Material(G.LAMBERT, color=(1.0, 1.0, 1.0)))     # dummy (DiffuseMaterial())
    masks.add()
    for name in obj.materials[1:]:
        mat = lib.get(name)
        mask_id = -1
        if mat is None:
            materials.append(G.Material(G.LAMBERT, color=(1.0, 1.0, 1.0)))
        else:
            if any(c > 0.0 for c in mat.ke):
                emissive[len(materials)] = mat.ke
            bump = tex.load(os.path.join(base, mat.map_bump)) if mat.map_bump else -1
            if mat.illum == 5:
                m = G.Material(G.MIRROR, color=mat.ks, eta=1.0, kappa=mat.ns, bump=bump)
            elif mat.illum == 7:
                m = G.Material(G.GLASS, color=mat.tf, specular=mat.ks, eta=mat.ni, bump=bump)
            else:
                kind = G.GLOSSY if any(c > 0.0 for c in mat.ks) else G.LAMBERT
                color, t = mat.kd, -1
                if mat.map_kd:
                    t = tex.load(os.path.join(base, mat.map_kd))
                    if t < 0:
                        color = (1.0, 0.0, 1.0)
                m = G.Material(kind, color=color, specular=mat.ks if kind == G.GLOSSY else (0.0, 0.0, 0.0),
                               exponent=mat.ns if kind == G.GLOSSY else 1.0, texture=t, bump=bump)
            materials.append(m)
            if mat.map_d:
                mask_id = tex.load(os.path.join(base, mat.map_d))
        if mask_id >= 0:
            if mask_id in mask_ids:
                masks.add(mask_ids[mask_id])
            else:
                mask_ids[mask_id] = masks.append(tex.images[mask_id])
        else:
            masks.add()


def _create_mesh(obj: ObjFile, materials: list, emissive: dict, mtl_offset: int, masks: _Masks):
    """create_mesh (build_scene.cpp:184-304): one mesh for the file."""
    verts = np.zeros((0, 3), np.float32)
    nrms = np.zeros((0, 3), np.float32)
    tcs = np.zeros((0, 2), np.float32)
    idx_all = np.zeros((0, 4), np.int32)
    tri_lights = []
    ov = np.asarray(obj.vertices, np.float32)
    on = np.asarray(obj.normals, np.float32)
    ot = np.asarray(obj.texcoords, np.float32)
    for groups in obj.objects:
        mapping, tris = {}, []
        has_n = has_t = False
        for faces in groups:
            for fidx, fmat in faces:
                for key in fidx:
                    if key not in mapping:
                        has_n |= key[2] != 0
                        has_t |= key[1] != 0
                        mapping[key] = len(mapping)
                v0 = mapping[fidx[0]]
                prev = mapping[fidx[1]]
                for i in range(1, len(fidx) - 1):
                    nxt = mapping[fidx[i + 1]]
                    m = fmat + mtl_offset
                    if m in emissive:
                        base = materials[m]
                        e = emissive[m]
                        dup = G.Material(G.EMISSIVE, color=base.color, specular=base.specular,
                                         exponent=base.exponent, eta=base.eta, kappa=base.kappa, emission=e,
                                         texture=base.texture, bump=base.bump)
                        materials.append(dup)
                        m = len(materials) - 1
                        masks.add()
                        p = [ov[fidx[0][0]], ov[fidx[i][0]], ov[fidx[i + 1][0]]]
                        tri_lights.append((p, e))
                    tris.append((v0, prev, nxt, m))
                    prev = nxt
        if not tris:
            continue
        off = len(verts)
        t = np.array(tris, np.int32)
        t[:, :3] += off
        idx_all = np.concatenate([idx_all, t])
        keys = list(mapping.keys())            # insertion order = the mapped index
        verts = np.concatenate([verts, ov[[k[0] for k in keys]]])
        tcs = np.concatenate([tcs, ot[[k[1] for k in keys]] if has_t else np.zeros((len(keys), 2), np.float32)])
        if has_n:
            nrms = np.concatenate([nrms, on[[k[2] for k in keys]]])
        else:
            # The reference recomputes the normals of the whole mesh built so far.
            nrms = np.concatenate([nrms, np.zeros((len(keys), 3), np.float32)])
            nrms = _compute_normals(verts, idx_all)
    gn = _normalize_rows(_face_cross(verts, idx_all)) if len(idx_all) else np.zeros((0, 3), np.float32)
    bad = np.isnan(nrms).any(1)
    nrms[bad] = (0.0, 1.0, 0.0)
    return verts, nrms, tcs, idx_all, gn, tri_lights


def load_scene_file(path: str, width: int = 512, height: int = 512, fov: float = 60.0) -> G.SceneDesc:
    """build_scene (build_scene.cpp:548-651) into a SceneDesc. The returned description
    carries `accel_files` (per-mesh cache files, for scene.build_traversal_data), `masks`
    and `mask_buffer` (opacity masks per material) and lists the file's directional, point
    and spot lights before the triangle lights, as the reference's light list has them."""
    info = parse_scene_file(path)
    materials, tex, masks, mask_ids = [], _Textures(), _Masks(), {}
    meshes, mesh_lights = [], []
    for mf in info.mesh_files:
        obj = parse_obj(mf)
        lib: dict = {}
        for name in obj.mtl_libs:
            parse_mtl(os.path.join(os.path.dirname(mf) or ".", name), lib)
        emissive: dict = {}
        mtl_offset = len(materials)
        _convert_materials(mf, obj, lib, materials, emissive, tex, masks, mask_ids)
        v, n, t, idx, gn, tl = _create_mesh(obj, materials, emissive, mtl_offset, masks)
        if len(idx) == 0:
            raise ValueError(f"scene: no triangle in {mf}")
        meshes.append(Mesh(v, idx, normals=n, texcoords=t, geom_normals=gn))
        mesh_lights.append(tl)
    instances, lights = [], []
    for mesh_id, mat in info.instances:
        if not 0 <= mesh_id < len(meshes):
            raise ValueError(f"scene: instance of unknown mesh {mesh_id}")
        instances.append(Instance(mesh_id, mat))
        for (p0, p1, p2), e in mesh_lights[mesh_id]:
            lights.append((_xform_point(mat, p0), _xform_point(mat, p1), _xform_point(mat, p2),
                           np.asarray(e, np.float32)))
    env_map, env_intensity = -1, 1.0
    if info.env is not None:
        img = load_hdr(info.env[0])
        env_map, env_intensity = len(tex.images), info.env[1]
        tex.images.append(img)
    if not lights and not info.lights and env_map < 0:
        raise ValueError("scene: there are no lights in the scene")
    cam = G.Camera(info.cam_pos, info.cam_dir, info.cam_up, fov, width, height)
    return G.SceneDesc(meshes, instances, materials, lights, cam, None, os.path.basename(path),
                       delta_lights=list(info.lights), textures=tex.images, delta_first=True,
                       masks=np.array(masks.descs, N.MASK_DTYPE), mask_buffer=np.concatenate(masks.buffer),
                       accel_files=info.accel_files, env_map=env_map, env_map_intensity=env_intensity)
