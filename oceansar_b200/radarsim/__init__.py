"""Radar simulation: the raw-data generator and its accumulation kernel."""
