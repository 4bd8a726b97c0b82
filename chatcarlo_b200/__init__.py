"""B200 photon-transport engine with ChatCarlo's transport interface."""
from .geometry import Geometry
from .scene import Scene, SceneError, load_scene, validate_scene
from .tally import VoxelGrid

__all__ = ["Geometry", "Scene", "SceneError", "VoxelGrid", "load_scene", "validate_scene",
           "transport_photons", "run_transport"]


def __getattr__(name):
    if name in ("transport_photons", "run_transport", "BatchResult", "TransportResult", "Engine"):
        from . import transport
        return getattr(transport, name)
    raise AttributeError(name)
