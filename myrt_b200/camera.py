"""Camera matrices in the form pt_generate.comp consumes them.

The reference builds its projection with rnu::cameraf (unvendored); callers of
this core pass the two inverse matrices directly. `look_at` returns a pair for
which (inverse_view @ inverse_projection @ (ndc_x, ndc_y, 1, 1)).xyz is the
view ray through that NDC point (w = 0, so the camera position does not leak
into the direction) and column 3 of inverse_view is the eye.
NDC y = -1 is image row 0 (GL texture convention).
"""
from __future__ import annotations

import numpy as np


def look_at(eye, target, up=(0.0, 1.0, 0.0), vfov_deg: float = 50.0, aspect: float = 1.0):
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    t = np.tan(np.radians(vfov_deg) / 2.0)
    inv_view = np.eye(4)
    inv_view[:3, 0], inv_view[:3, 1], inv_view[:3, 2], inv_view[:3, 3] = r, u, -f, eye
    inv_proj = np.zeros((4, 4))
    inv_proj[0, 0] = t * aspect
    inv_proj[1, 1] = t
    inv_proj[2, 3] = -1.0
    # column-major float32 arrays of 16, as the C ABI expects
    return (inv_view.T.astype(np.float32).ravel(), inv_proj.T.astype(np.float32).ravel())


def view_projection(eye, target, up=(0.0, 1.0, 0.0), vfov_deg: float = 50.0, aspect: float = 1.0,
                    near: float = 0.01, far: float = 100.0):
    """(view, projection) float32 [4, 4] in math layout for the forward
    renderer (forward_renderer::set_view_matrix / set_projection_matrix): a
    look-at view and the GL perspective matrix (clip z in [-w, w]). The ray of
    NDC (x, y) matches `look_at` with the same arguments."""
    eye = np.asarray(eye, np.float64)
    f = np.asarray(target, np.float64) - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, np.asarray(up, np.float64))
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    view = np.eye(4)
    view[0, :3], view[1, :3], view[2, :3] = r, u, -f
    view[:3, 3] = -view[:3, :3] @ eye
    t = np.tan(np.radians(vfov_deg) / 2.0)
    proj = np.zeros((4, 4))
    proj[0, 0] = 1.0 / (t * aspect)
    proj[1, 1] = 1.0 / t
    proj[2, 2] = -(far + near) / (far - near)
    proj[2, 3] = -2.0 * far * near / (far - near)
    proj[3, 2] = -1.0
    return view.astype(np.float32), proj.astype(np.float32)
