"""Writes viridis_table.h: the 256-entry viridis colour map as 8-bit RGB, for the command line's
FLIP --output image (FLIP value v is shown as entry floor(v * 255), as
shaders/flip/combine_error_maps.glsl:30-32 indexes its map).

The entries come from OpenCV's COLORMAP_VIRIDIS (cv2 4.13 here), which is matplotlib's viridis
rounded to 8 bits -- the same map the reference embeds as floats (src/gpu/flip/viridis.h), to within
that rounding.  Run it from this directory: python make_viridis.py
"""
import os

import cv2
import numpy as np

bgr = cv2.applyColorMap(np.arange(256, dtype=np.uint8).reshape(-1, 1), cv2.COLORMAP_VIRIDIS).reshape(256, 3)
rgb = bgr[:, ::-1]
lines = ["// Generated by make_viridis.py (OpenCV COLORMAP_VIRIDIS, 8-bit RGB); do not edit.",
         "#ifndef IQM_HOST_VIRIDIS_TABLE_H", "#define IQM_HOST_VIRIDIS_TABLE_H", "",
         "namespace IQM {", "inline constexpr unsigned char kViridisRGB[256][3] = {"]
for i in range(0, 256, 4):
    lines.append("    " + " ".join("{%d, %d, %d}," % tuple(int(c) for c in rgb[j]) for j in range(i, i + 4)))
lines += ["};", "}  // namespace IQM", "", "#endif", ""]
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "viridis_table.h")
with open(out, "w") as f:
    f.write("\n".join(lines))
