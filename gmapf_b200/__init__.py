"""B200-native G-MAPF per-frame step: bidirectional bounded-queue A* over a
navmesh triangle graph, path reconstruction, move-along-path and collision
avoidance, in hand-written CUDA for sm_100a behind the gmapf::GMAPF API."""
from .api import GMAPF, GMAPFError, EAgentState, SceneBatch, make_config, make_options, NODE_DTYPE, MODE_BATCHED, MODE_PLAIN  # noqa: F401
from . import _lib  # noqa: F401

__all__ = ["GMAPF", "GMAPFError", "EAgentState", "SceneBatch", "make_config", "make_options", "NODE_DTYPE",
           "MODE_BATCHED", "MODE_PLAIN"]
