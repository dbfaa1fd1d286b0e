"""Flat Barnes-Hut octree on the B200 (reference drop-in, FP64).

Drop-in for dem/octree/flat_tree.py:36-1630 of ddkx21/particle-simulator:
same constructor, parameters, attributes (``node_count[None]``,
``nodes.count.to_numpy()``, ...) and methods.  The tree is built and walked by
the CUDA kernels of libdem_b200 (csrc/tree.cu) with the reference's node
layout, numbering and summation order, so forces and velocities are
bit-identical to the reference's expressions in IEEE binary64.
"""

from __future__ import annotations

import weakref

import numpy as np

from .. import _native as N
from .._io import Stager
from ..periodic_correction.comsol_lattice_correction import correction_fields, to_device

_FIELDS_I32 = ("count", "first_child", "next", "leaf_start")


class _Scalar:
    """``field[None]`` access to a host-side scalar."""

    def __init__(self, getter, setter=None):
        self._get, self._set = getter, setter

    def __getitem__(self, key):
        return self._get()

    def __setitem__(self, key, value):
        if self._set is None:
            raise AttributeError("read-only field")
        self._set(value)


class _Field:
    """``.to_numpy()`` access to a device array (fetched on demand)."""

    def __init__(self, fetch):
        self._fetch = fetch

    def to_numpy(self):
        return self._fetch()

    def __getitem__(self, key):
        return self._fetch()[key]


class OctreeNode:
    """Node arrays of the tree (dem/octree/octree_node.py:12-154), read-only views."""

    def __init__(self, tree: "FlatOctree", max_nodes: int):
        ref = weakref.ref(tree)  # no reference cycle: the native handles are released in order
        self.max_nodes = max_nodes
        for name in _FIELDS_I32:
            setattr(self, name, _Field(lambda name=name: ref()._node_array(name)))
        for k, name in enumerate(("R3_sum", "R3_cx", "R3_cy", "R3_cz")):
            setattr(self, name, _Field(lambda k=k: ref()._node_array("r3")[:, k]))
        for k, name in enumerate(("force_sum_x", "force_sum_y", "force_sum_z", "fmom_xx", "fmom_xy", "fmom_xz",
                                  "fmom_yx", "fmom_yy", "fmom_yz", "fmom_zx", "fmom_zy", "fmom_zz")):
            setattr(self, name, _Field(lambda k=k: ref()._node_array("fs")[:, k]))


class FlatOctree:
    def __init__(self, theta: float = 0.5, mpl: int = 1, num_particles: int = 10000,
                 correction_grid_resolution: int = 0, *, device=None, max_nodes: int | None = None):
        self.theta = theta
        self.mpl = mpl
        n = max(num_particles, 64)  # flat_tree.py:63
        if max_nodes is None:
            max_nodes = max(4 * n // max(mpl, 1), 1024)  # :66
        self.max_nodes = max_nodes
        self.max_leaf_slots = n
        self.correction_grid_resolution = correction_grid_resolution
        self._ctx = N.Context(n, device)
        self._io = Stager(self._ctx)
        self._tree = N.Tree(self._ctx, n, max_nodes)
        self._n = 0
        self._L = 0.0
        self._periodic = 0
        self._theta_sq = theta * theta
        me = weakref.ref(self)  # field views must not keep the tree alive (no reference cycles)

        def _set_theta_sq(v):
            me()._theta_sq = float(v)

        def _set_mpl(v):
            me().mpl = int(v)

        self.theta_sq = _Scalar(lambda: me()._theta_sq, _set_theta_sq)
        self.mpl_field = _Scalar(lambda: me().mpl, _set_mpl)
        self.node_count = _Scalar(lambda: me()._tree.stats()["node_count"])
        self.parent_count = _Scalar(lambda: me()._tree.stats()["parent_count"])
        self.leaf_slot_count = _Scalar(lambda: me()._tree.stats()["leaf_slot_count"])
        self.num_particles = _Scalar(lambda: me()._n)
        self.L = _Scalar(lambda: me()._L)
        self.periodic = _Scalar(lambda: me()._periodic)
        self.nodes = OctreeNode(self, max_nodes)
        self.leaf_indices = _Field(lambda: me()._leaf_indices())
        self._F = None  # device SoA forces of the last force walk
        self._corr = None  # device grid of the periodic-image correction
        self.__dict__.update(correction_fields(None))

    # -- parameters (flat_tree.py:169-174) ------------------------------------
    def update_params(self, theta: float, mpl: int) -> None:
        self.theta = theta
        self.mpl = mpl
        self._theta_sq = theta * theta

    def load_periodic_correction(self, correction, L_sim: float, eta_sim: float = None):
        """flat_tree.py:141-167: the velocity walks add the correction from now on."""
        if self.correction_grid_resolution == 0:
            raise RuntimeError("correction_grid_resolution=0: correction grids were not allocated.")
        self._corr, scalars = to_device(self._ctx, correction, L_sim, eta_sim,
                                        max(self.correction_grid_resolution, 2))
        self._tree.set_correction(self._corr)
        self.__dict__.update(correction_fields(scalars))

    # -- build ----------------------------------------------------------------
    def build(self, positions, radii, L: float, periodic: bool = False):
        """flat_tree.py:180-246 (ValueError when n exceeds the capacity)."""
        n = len(radii)
        if n > self.max_leaf_slots:
            raise ValueError(
                f"Number of particles ({n}) exceeds allocated capacity ({self.max_leaf_slots}). "
                f"Recreate FlatOctree with larger num_particles.")
        st, _ = self._io.positions(positions, radii)
        self.build_soa(n, st.pos, st.r, L, periodic)

    def build_soa(self, n, pos_soa, r, L, periodic):
        self._n = n
        self._L = float(L)
        self._periodic = 1 if periodic else 0
        self._tree.build(n, pos_soa, r, self._L, self._periodic, self.mpl)

    # -- walks ----------------------------------------------------------------
    def _forces_dev(self, m_const):
        F = self._io.buf.dev("tree_F", (3, self._n))
        self._tree.forces(m_const, self._theta_sq, F)
        self._F = F
        return F

    def compute_forces(self, m_const: float) -> np.ndarray:
        """flat_tree.py:896-906."""
        if self._n == 0:
            return np.zeros((0, 3))
        return self._io.download([self._forces_dev(m_const)], self._n)[0]

    def _velocity_dev(self, F_soa, eta_const, stokes_factor, from_fields: bool):
        if from_fields:
            self._tree.propagate_forces(None)
        else:
            self._tree.propagate_forces(F_soa)
        V = self._io.buf.dev("tree_V", (3, self._n))
        self._tree.velocity(F_soa, eta_const, self._theta_sq, stokes_factor, V)
        return V

    def _forces_arg(self, forces):
        return self._io.vectors(forces, self._n, "tree_forces_in")

    def compute_stokeslet(self, forces, eta_const: float) -> np.ndarray:
        """flat_tree.py:1282-1294: moments from ``forces``."""
        F = self._forces_arg(forces)
        return self._io.download([self._velocity_dev(F, eta_const, 0.0, False)], self._n)[0]

    def compute_stokeslet_from_fields(self, forces, eta_const: float) -> np.ndarray:
        """flat_tree.py:1296-1312: moments from the forces of the last force walk."""
        F = self._forces_arg(forces)
        return self._io.download([self._velocity_dev(F, eta_const, 0.0, True)], self._n)[0]

    def compute_forces_and_stokeslet(self, m_const: float, eta_const: float) -> tuple:
        """flat_tree.py:1314-1324."""
        F = self._forces_dev(m_const)
        V = self._velocity_dev(F, eta_const, 0.0, True)
        f, v = self._io.download([F, V], self._n)
        return f, v

    def compute_total_velocity(self, forces, eta_const: float, stokes_factor: float) -> np.ndarray:
        """flat_tree.py:1590-1604."""
        F = self._forces_arg(forces)
        return self._io.download([self._velocity_dev(F, eta_const, stokes_factor, True)], self._n)[0]

    def compute_forces_and_total_velocity(self, m_const: float, eta_const: float, stokes_factor: float) -> tuple:
        """flat_tree.py:1606-1612."""
        F = self._forces_dev(m_const)
        V = self._velocity_dev(F, eta_const, stokes_factor, True)
        f, v = self._io.download([F, V], self._n)
        return f, v

    def total_velocity_soa(self, m_const, eta_const, stokes_factor):
        """Device-resident forces + total velocity (SoA device tensors)."""
        F = self._forces_dev(m_const)
        return F, self._velocity_dev(F, eta_const, stokes_factor, True)

    # -- diagnostics (flat_tree.py:1618-1630) ------------------------------------
    def get_tree_stats(self) -> dict:
        s = self._tree.stats()
        nc = s["node_count"]
        return {
            "node_count": nc,
            "max_nodes": self.max_nodes,
            "node_utilization": nc / self.max_nodes if self.max_nodes > 0 else 0.0,
            "parent_count": s["parent_count"],
            "num_particles": self._n,
            "leaf_slot_count": s["leaf_slot_count"],
        }

    def _node_array(self, name):
        torch = self._ctx.torch
        nc = self._tree.stats()["node_count"]
        if name in _FIELDS_I32:
            out = torch.empty(max(nc, 1), dtype=torch.int32, device=self._ctx.device)
            self._tree.nodes(**{("next_" if name == "next" else name): out})
        elif name == "r3":
            out = torch.empty((max(nc, 1), 4), dtype=torch.float64, device=self._ctx.device)
            self._tree.nodes(r3=out)
        else:
            out = torch.empty((max(nc, 1), 12), dtype=torch.float64, device=self._ctx.device)
            self._tree.nodes(fs=out)
        return out[:nc].cpu().numpy()

    def _leaf_indices(self):
        torch = self._ctx.torch
        out = torch.empty(max(self._n, 1), dtype=torch.int32, device=self._ctx.device)
        self._tree.leaf_indices(out)
        return out[: self._n].cpu().numpy()
