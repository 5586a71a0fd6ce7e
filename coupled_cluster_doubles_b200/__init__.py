"""B200-native drop-in for the CCD T2 iteration of justinlietz/coupled_cluster_doubles."""
from .system import System  # noqa: F401
