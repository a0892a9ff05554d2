"""Ocean surfaces (``oceansar/surfaces``): ``OceanSurface`` with fields synthesised on the GPU."""
from .ocean import OceanSurface  # noqa: F401
