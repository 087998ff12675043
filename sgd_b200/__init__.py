"""B200-native CT projector layer with the interface of hqpwca/SGD's projectors.

Forward and back (adjoint) projectors as hand-written sm_100a CUDA kernels in
``libnetwork.so`` behind the reference's C entry points; ``operators`` mirrors
the reference's Python LinearOperator wrappers (python/operators/operators.py)
and ``torch_ops`` exposes the same kernels on device tensors.
"""
from ._lib import LIB_PATH, ProjectorError  # noqa: F401

__all__ = ["LIB_PATH", "ProjectorError"]
