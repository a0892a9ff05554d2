"""The DopSCA scatterometer raw-data generator (``oceansar/dopscasim``) on the GPU."""
from .dopsca_raw import DopscaGenerator, dopsca_raw  # noqa: F401
