"""B200-native embedding-extension engine with the capabilities of Khuzdul's counting path.

The engine is libkhz_b200.so (CUDA for sm_100a behind the C ABI in include/khz.h);
`khz` is its Python binding.
"""
from . import khz  # noqa: F401
from .khz import APPS, Context, Graph, KhzError, num_counts, set_op_batch  # noqa: F401
