"""Seeded synthetic textures with the shapes and value distributions of the benchmark workloads.

The reference measures on photographs that are not available here; these generators stand in for them. Every
function is deterministic for a given seed and device (torch.Generator), and the parity tests always hand the exact
generated bytes to both the GPU encoder and the CPU oracle, so the content itself needs no cross-device bit-exactness.

  colour_texture  - sum of 3 smooth colour gradients + 4-octave value noise (amplitude 0.3) + 20 hard-edged
                    axis-aligned rectangles of uniform random colour, quantised to RGBA8 (alpha 255, or noise alpha
                    thresholded at 30% to 0 and otherwise smooth)
  normal_map      - RG8 tangent-space normals from a 5-octave fBm heightfield (Sobel gradient, normalised)
  hdr_texture     - RGB16F: log2(luminance) uniform in [-8, 8] from 3-octave noise, hue from smooth gradients,
                    50 Gaussian highlights up to 2^12
  batch_sizes     - power-of-two sides 64..2048, log-uniform, aspect <= 4:1
"""
import math

import torch
import torch.nn.functional as F


def _gen(seed, device):
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) & 0x7FFFFFFFFFFFFFFF)
    return g


def _cells(w, h, finest_period_octaves_scale):
    """Lattice cells of the base octave so that detail scales with the texture: for the 4-octave colour noise
    (scale 64) the finest octave has a period of 8 texels, i.e. block-scale detail like a photograph's."""
    return max(2, min(w, h) // finest_period_octaves_scale)


def value_noise(h, w, octaves, base_cells, g, device, channels=1, persistence=0.5):
    """Sum of `octaves` lattice value-noise layers (bicubic-interpolated lattices), normalised to [0, 1]."""
    out = torch.zeros(channels, h, w, device=device)
    amp, total = 1.0, 0.0
    cells = base_cells
    for _ in range(octaves):
        lat = torch.rand(1, channels, cells + 1, cells + 1, generator=g, device=device)
        layer = F.interpolate(lat, size=(h, w), mode="bicubic", align_corners=True)[0]
        out += amp * layer
        total += amp
        amp *= persistence
        cells *= 2
    return (out / total).clamp_(0, 1)


def _gradients(h, w, n, g, device):
    y = torch.linspace(0, 1, h, device=device).view(h, 1)
    x = torch.linspace(0, 1, w, device=device).view(1, w)
    acc = torch.zeros(3, h, w, device=device)
    for _ in range(n):
        theta = float(torch.rand(1, generator=g, device=device)) * 2 * math.pi
        col = torch.rand(3, generator=g, device=device).view(3, 1, 1)
        ramp = (x * math.cos(theta) + y * math.sin(theta))
        ramp = (ramp - ramp.min()) / (ramp.max() - ramp.min() + 1e-9)
        acc += col * ramp
    return acc / n


def colour_texture(w, h, seed=0, alpha="opaque", device="cpu"):
    """HxWx4 uint8. alpha: "opaque" (255) or "noise" (2-octave noise, thresholded at 30% to 0, else smooth)."""
    g = _gen(seed, device)
    img = _gradients(h, w, 3, g, device)
    img = img * 0.7 + 0.3 * value_noise(h, w, 4, _cells(w, h, 64), g, device, channels=3)
    for _ in range(20):
        rw = int(torch.randint(max(1, w // 32), max(2, w // 4), (1,), generator=g, device=device))
        rh = int(torch.randint(max(1, h // 32), max(2, h // 4), (1,), generator=g, device=device))
        x0 = int(torch.randint(0, max(1, w - rw), (1,), generator=g, device=device))
        y0 = int(torch.randint(0, max(1, h - rh), (1,), generator=g, device=device))
        img[:, y0:y0 + rh, x0:x0 + rw] = torch.rand(3, 1, 1, generator=g, device=device)
    rgba = torch.empty(h, w, 4, dtype=torch.uint8, device=device)
    rgba[..., :3] = (img.clamp(0, 1) * 255 + 0.5).to(torch.uint8).permute(1, 2, 0)
    if alpha == "opaque":
        rgba[..., 3] = 255
    else:
        a = value_noise(h, w, 2, _cells(w, h, 32), g, device)[0]
        a = torch.where(a < 0.3, torch.zeros_like(a), (a - 0.3) / 0.7)
        rgba[..., 3] = (a * 255 + 0.5).to(torch.uint8)
    return rgba


def normal_map(w, h, seed=0, device="cpu"):
    """HxWx2 uint8 tangent-space normal xy (unorm8) from a 5-octave fBm heightfield."""
    g = _gen(seed, device)
    hf = value_noise(h + 2, w + 2, 5, _cells(w, h, 128), g, device)[0] * 32.0
    p = hf.view(1, 1, h + 2, w + 2)
    kx = torch.tensor([[-1.0, 0, 1], [-2, 0, 2], [-1, 0, 1]], device=device).view(1, 1, 3, 3) / 8
    gx = F.conv2d(p, kx)[0, 0]
    gy = F.conv2d(p, kx.transpose(2, 3))[0, 0]
    n = torch.stack([-gx, -gy, torch.ones_like(gx)], 0)
    n = n / n.norm(dim=0, keepdim=True)
    out = ((n[:2] * 0.5 + 0.5).clamp(0, 1) * 255 + 0.5).to(torch.uint8).permute(1, 2, 0)
    return out.contiguous()


def hdr_texture(w, h, seed=0, device="cpu"):
    """HxWx3 float16 (non-negative, finite)."""
    g = _gen(seed, device)
    l2 = value_noise(h, w, 3, _cells(w, h, 64), g, device)[0]
    l2 = (l2 - l2.min()) / (l2.max() - l2.min() + 1e-9) * 16.0 - 8.0  # log2 luminance spread over [-8, 8]
    hue = _gradients(h, w, 2, g, device) * 0.8 + 0.2
    lum = torch.exp2(l2)
    y = torch.arange(h, device=device, dtype=torch.float32).view(h, 1)
    x = torch.arange(w, device=device, dtype=torch.float32).view(1, w)
    for _ in range(50):
        cx, cy = float(torch.rand(1, generator=g, device=device)) * w, float(torch.rand(1, generator=g, device=device)) * h
        sig = 1.0 + float(torch.rand(1, generator=g, device=device)) * max(w, h) / 64
        peak = 2.0 ** (float(torch.rand(1, generator=g, device=device)) * 12)
        lum = lum + peak * torch.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * sig * sig))
    rgb = (hue * lum.unsqueeze(0)).clamp(0, 65504.0)
    return rgb.permute(1, 2, 0).to(torch.float16).contiguous()


def batch_sizes(n, seed=0, lo=6, hi=11, max_aspect_log2=2):
    """n (w, h) pairs: log2 sides uniform in [lo, hi], |log2 w - log2 h| <= max_aspect_log2 (aspect <= 4:1)."""
    g = torch.Generator()
    g.manual_seed(seed)
    out = []
    while len(out) < n:
        a, b = torch.randint(lo, hi + 1, (2,), generator=g).tolist()
        if abs(a - b) <= max_aspect_log2:
            out.append((1 << a, 1 << b))
    return out


def batch_formats(n, seed=0, mix=((0, 0.4), (1, 0.2), (4, 0.4))):
    """n format ids drawn with the given (format, probability) mix (default 40% BC1, 20% BC3, 40% BC7)."""
    g = torch.Generator()
    g.manual_seed(seed + 1)
    u = torch.rand(n, generator=g).tolist()
    fmts = []
    for v in u:
        acc = 0.0
        for f, p in mix:
            acc += p
            if v < acc:
                fmts.append(f)
                break
        else:
            fmts.append(mix[-1][0])
    return fmts
