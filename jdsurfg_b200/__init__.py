"""jdsurfg_b200: B200-native surface-wave dispersion and depth kernels for
JDSurfG's SurfTime path (libswdk.so + thin Python binding)."""
from .engine import Engine, SwdkError, ST_OK, ST_NO_ROOT, ST_RETRIED, ST_NAN_INPUT, ST_ITER_LIMIT  # noqa: F401
