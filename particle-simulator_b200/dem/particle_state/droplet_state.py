"""Droplet state container, mirroring dem/particle_state/droplet_state.py:7-100
of the reference: positions (N, 3), radii (N,), time; npz and xlsx I/O."""

from __future__ import annotations

import numpy as np


class DropletState:
    def __init__(self, positions=None, radii=None, time=0, filename=None):
        self.positions = None
        self.radii = None
        self.time = 0
        if positions is not None and radii is not None:
            self.positions = np.array(positions)
            self.radii = np.array(radii)
            self.time = time
        elif filename is not None:
            if filename.endswith(".xlsx"):
                self.import_from_xlsx(filename)
            elif filename.endswith(".npz"):
                self.load(filename)
            else:
                raise ValueError("the file must have a .xlsx or .npz extension")
        else:
            raise ValueError("pass either positions and radii, or a file name")

    def copy(self):
        return DropletState(self.positions.copy(), self.radii.copy(), self.time)

    def save(self, filename):
        np.savez(filename, positions=self.positions, radii=self.radii, time=self.time)

    def load(self, filename):
        data = np.load(filename)
        self.positions = data["positions"]
        self.radii = data["radii"]
        self.time = float(data["time"])

    def export_to_xlsx(self, filename):
        import pandas as pd

        df = pd.DataFrame({"x": self.positions[:, 0], "y": self.positions[:, 1], "z": self.positions[:, 2], "r": self.radii})
        df.to_excel(filename, index=False)

    def import_from_xlsx(self, filename):
        import pandas as pd

        df = pd.read_excel(filename)
        self.positions = np.array(df[["x", "y", "z"]])
        self.radii = np.array(df["r"])
        self.time = 0

    def __repr__(self):
        return f"<DropletState: time={self.time}, num_particles={len(self.radii)}>"
