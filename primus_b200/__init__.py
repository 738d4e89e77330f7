"""primus_b200: B200-native (sm_100a) backend for the primus lattice-arithmetic path.

The compute lives in libprimus_gpu.so (hand-written CUDA, C ABI in
include/primus_gpu.h); this package is the host-side mirror of the reference's
trait API.  Importing it loads the library and fails loudly when it is absent.
"""
from ._native import (DeviceBuffer, Event, PrimusGpuError, Stream, device_count, launch_count,  # noqa: F401
                      synchronize)
from .lattice import (BaseConverter, GadgetBasis, RnsBase, RnsError, external_product,  # noqa: F401
                      external_product_coeff, HybridKeySwitch, glwe_automorphism, glwe_trace,
                      glwe_expand_coefficients, BfvDecryptor, GlweEncryptor,
                      ext_product_workspace_size, glev_mac_big_uint_poly, glev_mac_crt_poly, key_switch,
                      key_switch_workspace_size)
from .server import (Request, Server, ext_product_request, key_switch_request,  # noqa: F401
                     polymul_request)
from .ntt import (DcrtTable, NttError, NttTable, PolymulBatch, host_tables, minimal_primitive_root,  # noqa: F401
                  ntt_primes, prev_prime_congruent, variant_count, variant_name, calibrate)

__all__ = [
    "DcrtTable", "NttTable", "NttError", "DeviceBuffer", "Stream", "Event", "PrimusGpuError",
    "ntt_primes", "prev_prime_congruent", "minimal_primitive_root", "host_tables", "device_count",
    "launch_count", "synchronize", "RnsBase", "RnsError", "BaseConverter", "GadgetBasis", "external_product",
    "ext_product_workspace_size", "glev_mac_crt_poly", "glev_mac_big_uint_poly", "key_switch", "PolymulBatch", "Server", "Request",
    "polymul_request", "ext_product_request", "key_switch_request", "external_product_coeff",
    "key_switch_workspace_size", "HybridKeySwitch", "glwe_automorphism", "glwe_trace", "glwe_expand_coefficients",
    "BfvDecryptor", "GlweEncryptor", "variant_count", "variant_name",
]
