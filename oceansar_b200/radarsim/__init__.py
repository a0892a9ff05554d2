"""Radar simulation: the raw-data generators (``sar_raw_nompi``, the time-interpolated
``sar_raw.sarraw``, ``skim_raw``), their accumulation kernel (``range_profile``), the scene
batch and the range-Doppler processor (``sar_processor``)."""
