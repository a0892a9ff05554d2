"""Ocean surfaces (``oceansar/surfaces``): ``OceanSurface`` with fields synthesised on the GPU,
and ``OceanSurfaceBalancer``, its time-interpolated form."""
from .balancer import OceanSurfaceBalancer  # noqa: F401
from .ocean import OceanSurface  # noqa: F401
