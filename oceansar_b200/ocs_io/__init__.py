"""Configuration and file I/O (``oceansar/ocs_io``): the ``.cfg`` reader and the raw /
ocean-state files (``.npz`` containers with the reference's variable names)."""
from .cfg import ConfigFile  # noqa: F401
