"""ctypes signatures of the oracle's optional entry points (test infrastructure only)."""
import ctypes as C

vp, u64, i32, f32, f64 = C.c_void_p, C.c_uint64, C.c_int, C.c_float, C.c_double

SIGNATURES: dict = {}
