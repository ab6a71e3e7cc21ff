"""FEField: the ndarray subclass solve_static returns (fields.py:36), reduced to what the
static path needs: named DOF components and nodal reshaping."""
from __future__ import annotations

import numpy as np


class FEField(np.ndarray):
    def __new__(cls, data, n_nodes, dofs_per_node=3, dof_names=("ux", "uy", "uz"), label=None, mesh=None):
        obj = np.asarray(data, dtype=float).view(cls)
        obj.n_nodes = int(n_nodes)
        obj.dofs_per_node = int(dofs_per_node)
        obj.dof_names = tuple(dof_names)
        obj.label = label
        obj.mesh = mesh
        return obj

    def __array_finalize__(self, obj):
        if obj is None:
            return
        self.n_nodes = getattr(obj, "n_nodes", None)
        self.dofs_per_node = getattr(obj, "dofs_per_node", 3)
        self.dof_names = getattr(obj, "dof_names", ("ux", "uy", "uz"))
        self.label = getattr(obj, "label", None)
        self.mesh = getattr(obj, "mesh", None)

    @property
    def nodal(self):
        """(n_nodes, dofs_per_node) view of a full DOF vector."""
        return np.asarray(self).reshape(self.n_nodes, self.dofs_per_node)

    def component(self, name, nodes=None):
        k = self.dof_names.index(name) if isinstance(name, str) else int(name)
        vals = self.nodal[:, k]
        if nodes is None:
            return vals
        if isinstance(nodes, str):
            if self.mesh is None or nodes not in getattr(self.mesh, "node_sets", {}):
                raise ValueError(f"unknown node set {nodes!r}")
            nodes = self.mesh.node_sets[nodes]
        return vals[np.asarray(nodes, dtype=int)]

    def magnitude(self):
        return np.linalg.norm(self.nodal, axis=1)
