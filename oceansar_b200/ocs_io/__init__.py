"""Configuration and file I/O (``oceansar/ocs_io``): the ``.cfg`` reader, and the raw and
ocean-state files in the netCDF classic format (``netcdf3``)."""
from .cfg import ConfigFile  # noqa: F401
from .netcdf import NETCDFHandler  # noqa: F401
from .processed import ProcFile  # noqa: F401
from .raw import DopscaRawFile, RawFile, SkimRawFile  # noqa: F401
from .state import OceanStateFile  # noqa: F401
