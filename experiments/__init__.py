"""Experiment harness over the imops_b200 adjoint C-ABI (torch autograd,
parameter fitting, data-parallel gradient reduction)."""
