"""CPU oracle of the headless colour-map export (test infrastructure only: the tests compare
fip_render's CUDA output with it; nothing in the product calls it).

Restates the reference's fragment shader (src/shaders.h:57-123) for a view from straight above:
  * src/shaders.h:57-83  colormap_red/green/blue/jet (MATLAB jet, clamped to [0, 1]);
  * src/shaders.h:93-96  depth > 1 cm: jet(min(1, depth / maxDepth));
  * src/shaders.h:98-105 velocity: qx / max(0.01, (h + h_east) / 2), qy / max(0.01, (h + h_north)
    / 2), speed, jet(min(1, speed / maxVelocity));
  * src/shaders.h:88-90  terrain == no_data (the vertex shader's Valid = 0): transparent;
  * src/shaders.h:108-123 dry cells: normal = normalize(hL - hR, 2, hD - hU), light
    normalize(1, -5, 1), 0.15 + 0.55 max(0, n.-l) + 0.3 max(0, v.reflect(l, n))^4, white;
    the eye straight above gives v = (0, 1, 0).
Texture reads clamp at the edges (GL_CLAMP_TO_EDGE, src/vis.cpp:209-210). Output rows are north
first (grid row H-1 first). FP64 arithmetic; the GPU result must agree within one 8-bit step.
"""
import numpy as np


def _jet(x):
    r = np.clip(np.where(x < 0.7, 4.0 * x - 1.5, -4.0 * x + 4.5), 0.0, 1.0)
    g = np.clip(np.where(x < 0.5, 4.0 * x - 0.5, -4.0 * x + 3.5), 0.0, 1.0)
    b = np.clip(np.where(x < 0.3, 4.0 * x + 0.5, -4.0 * x + 2.5), 0.0, 1.0)
    return r, g, b


def render(h, qx, qy, terrain, no_value, what="depth", vmax=5.0):
    h = np.asarray(h, np.float64)
    t = np.asarray(terrain, np.float64)
    H, W = h.shape
    ce = np.minimum(np.arange(W) + 1, W - 1)
    cw = np.maximum(np.arange(W) - 1, 0)
    rn = np.minimum(np.arange(H) + 1, H - 1)
    rs = np.maximum(np.arange(H) - 1, 0)
    if what == "velocity":
        ux = np.asarray(qx, np.float64) / np.maximum(0.01, (h + h[:, ce]) * 0.5)
        uy = np.asarray(qy, np.float64) / np.maximum(0.01, (h + h[rn, :]) * 0.5)
        v = np.sqrt(ux * ux + uy * uy)
    else:
        v = h
    x = np.minimum(1.0, v / vmax)
    r, g, b = _jet(x)
    nx, ny, nz = t[:, cw] - t[:, ce], np.full_like(t, 2.0), t[rs, :] - t[rn, :]
    nl = np.sqrt(nx * nx + ny * ny + nz * nz)
    nx, ny, nz = nx / nl, ny / nl, nz / nl
    l = np.array([1.0, -5.0, 1.0]) / np.sqrt(27.0)
    d = nx * l[0] + ny * l[1] + nz * l[2]
    ry = l[1] - 2.0 * d * ny
    shade = np.clip(0.15 + 0.55 * np.maximum(0.0, -d) + 0.3 * np.maximum(0.0, ry) ** 4, 0.0, 1.0)
    wet = h > 0.01
    out = np.zeros((H, W, 4), np.float64)
    out[..., 0] = np.where(wet, r, shade)
    out[..., 1] = np.where(wet, g, shade)
    out[..., 2] = np.where(wet, b, shade)
    out[..., 3] = 1.0
    out[t == no_value] = 0.0
    return np.rint(out * 255.0)[::-1].astype(np.int32)
