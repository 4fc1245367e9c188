"""Vertical staggering (oracle_v8/grid/__init__.py)."""
from .staggering import CharneyPhillipsStaggering, GridStaggering, LevelType, LorenzStaggering

__all__ = ["GridStaggering", "LorenzStaggering", "CharneyPhillipsStaggering", "LevelType"]
