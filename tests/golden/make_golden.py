"""Regenerates the committed golden fixtures from a reference checkout.

    python tests/golden/make_golden.py <path of the reference checkout>

It copies the reference's own pyFAI-derived geometry vectors
(test_data/test_reference/*_pyFAI.txt, for test_data/v1.poni on a 10 x 20
detector; the reference compares them in src/geometry.rs:789-920) and the
v1.poni calibration into tests/golden/geometry_v1.npz, so the tests need no
reference checkout at run time.
"""
import os
import sys

import numpy as np

NAMES = ["x_pyFAI", "y_pyFAI", "z_pyFAI", "tth_pyFAI", "azimuth_pyFAI",
         "solid_angle_pyFAI", "polarization_pyFAI", "d1_cart_poni", "d2_cart_poni"]
PONI_KEYS = {"PixelSize1": "pixel1", "PixelSize2": "pixel2", "Distance": "distance",
             "Poni1": "poni1", "Poni2": "poni2", "Rot1": "rot1", "Rot2": "rot2",
             "Rot3": "rot3", "Wavelength": "wavelength"}


def main(ref: str) -> None:
    data = {}
    for name in NAMES:
        path = os.path.join(ref, "test_data", "test_reference", name + ".txt")
        with open(path) as f:
            data[name] = np.array([float(line) for line in f if line.strip()], np.float64)
    poni = {}
    with open(os.path.join(ref, "test_data", "v1.poni")) as f:
        for line in f:
            if line.startswith("#") or ":" not in line:
                continue
            key, value = (s.strip() for s in line.split(":", 1))
            if key in PONI_KEYS:
                poni[PONI_KEYS[key]] = float(value)
    for k, v in poni.items():
        data["poni_" + k] = np.array(v)
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "geometry_v1.npz")
    np.savez(out, **data)
    print("wrote", out, sorted(data))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
