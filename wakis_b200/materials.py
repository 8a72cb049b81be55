"""Material library: key -> [eps_r, mu_r(, sigma [S/m])].

Same keys and values as upstream (wakis/materials.py:27-62).
"""

import numpy as np

material_lib = {
    "pec": [np.inf, 1.0],
    "vacuum": [1.0, 1.0],
    "dielectric": [10.0, 1.0],
    "lossy metal": [10, 1.0, 10],
    "copper": [5.8e07, 1.0, 5.8e07],
    "berillium": [2.5e07, 1.0, 2.5e07],
    "stainless steel": [1.4e06, 1.0, 1.4e06],
}

material_colors = {
    "pec": "white",
    "vacuum": "tab:blue",
    "dielectric": "tab:green",
    "lossy metal": "tab:orange",
    "copper": [0.82745099, 0.698039, 0.49019599],
    "berillium": [0.82745099, 0.698039, 0.49019599],
    "stainless steel": "silver",
    "martensite": [0.0, 1.0, 1.0],
    "other": "cyan",
}


def resolve(mat):
    """Library key or explicit list -> [eps_r, mu_r(, sigma)]."""
    if isinstance(mat, str):
        lib = material_lib[mat.lower()]
        return [lib[0], lib[1]] + ([lib[2]] if len(lib) == 3 else [])
    return list(mat)
