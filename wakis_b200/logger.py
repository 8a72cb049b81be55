"""Run log (upstream wakis/logger.py:13-97): grid / solver / wakeSolver
dicts written as JSON to ``<folder>/wakis.log``."""

import json
import os

import numpy as np


class Logger:
    def __init__(self):
        self.grid = {}
        self.solver = {}
        self.wakeSolver = {}

    def save_logs(self, folder="results/"):
        if not folder.endswith("/"):
            folder += "/"
        os.makedirs(folder, exist_ok=True)

        def conv(v):
            if isinstance(v, np.ndarray):
                return v.tolist()
            if isinstance(v, (np.floating, np.integer)):
                return v.item()
            if isinstance(v, (list, tuple)):
                return [conv(x) for x in v]
            if isinstance(v, dict):
                return {str(k): conv(x) for k, x in v.items()}
            if isinstance(v, (str, int, float, bool)) or v is None:
                return v
            return str(v)

        with open(folder + "wakis.log", "w") as f:
            json.dump({"grid": conv(self.grid), "solver": conv(self.solver),
                       "wakeSolver": conv(self.wakeSolver)}, f, indent=2)
