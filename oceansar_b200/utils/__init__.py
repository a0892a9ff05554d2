"""Host utilities: geometry and FFT sizes (``oceansar/utils``)."""
from .misc import optimize_fftsize, db, db2lin  # noqa: F401
