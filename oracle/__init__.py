"""Oracle: CPU restatement of the OCEANSAR raw-data-generation path.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline / reference legs may import anything from this package, and
only as the checker or the timed CPU baseline.  The product package ``oceansar_b200``
never imports it and has no CPU fallback.

Parity status: PINNED.  Every function here is checked (``tests/test_oracle_golden.py``)
against fixtures under ``tests/golden/`` that were produced by running the unmodified
reference code itself (``tests/golden/make_golden.py``): the numba accumulator, the
surface fields, the Romeiser Bragg RCS, the Kodis field, the closure series, the
geometry helpers, the ``.cfg`` parser and three end-to-end ``sar_raw`` runs.

Modules (each function cites the reference ``file:line`` it restates):

* ``range_profile``  -- sinc table + facet-to-range-bin accumulation (C, ``range_profile.c``)
* ``spectra``        -- Elfouhaily spectrum / spreading, cos^2 spreading, Ardhuin swell
* ``surface``        -- ``OceanSurface`` init and per-time field synthesis (numpy FFT)
* ``nrcs``           -- Romeiser'97 Bragg RCS and Kodis specular field
* ``closure``        -- coherence time and random sub-grid scatterer series
* ``geometry``       -- spherical-Earth geometry and ``optimize_fftsize``
* ``cfg``            -- ``.cfg`` reader
* ``sar_raw``        -- the per-pulse raw generation loop
"""
