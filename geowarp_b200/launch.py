"""Vectorised stand-in for wp.launch of the user boundary-condition kernels.

The reference's problem scripts write Warp kernels that set Dirichlet flags
(e.g. problems/bar_compaction/bar_compaction_cpGIMP.py:93-107) and launch them
over the node lattice with wp.launch(kernel, dim=(nx+1, ny+1), inputs=[...]).
Here the same "kernel" is a Python function that receives the launch indices
as integer tensors (one per launch dimension, all threads at once) followed by
the inputs, and writes flags with tensor indexing:

    def set_boundary_dofs(tid, boundary_flag_array, n_grid_x, n_nodes):
        node_idx, node_idy = tid
        dof_x = node_idx + node_idy * (n_grid_x + 1)
        boundary_flag_array[dof_x[(node_idx <= 1) | (node_idx >= 2)]] = True
"""
import torch


def launch(kernel, dim, inputs, device=None):
    """Call kernel(tid, *inputs) with tid = index tensors over the launch grid."""
    if device is None:
        device = next((t.device for t in inputs if isinstance(t, torch.Tensor)), torch.device("cpu"))
    if isinstance(dim, int):
        tid = torch.arange(dim, device=device)
        return kernel(tid, *inputs)
    axes = [torch.arange(int(d), device=device) for d in dim]
    grids = torch.meshgrid(*axes, indexing="ij")
    tid = tuple(g.reshape(-1) for g in grids)
    return kernel(tid, *inputs)
