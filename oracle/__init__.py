"""CPU oracle for the rcabeam OPW path -- TEST INFRASTRUCTURE ONLY.

This package restates, in float64 / complex128 NumPy, the reference algorithm
of sdiebolt/rcabeam for the OPW path:

* ``das``      -- RC/CR delay-and-sum (src/rcabeam/sim.py:344-393), angle and
                  aperture compounding (src/rcabeam/opw.py:8-21) and power
                  Doppler (src/rcabeam/power.py:8-21);
* ``methods``  -- the batching-form methods XDoppler (xdoppler.py:33-51) and
                  DMAS-CCF-ACF (dmas.py:32-85), evaluated per frame;
* ``clutter``  -- the global temporal SVD clutter filter
                  (src/rcabeam/clutter.py:10-109) in complex128;
* ``adjoint``  -- the float64 adjoint of the DAS forward model;
* ``c_das``    -- the same float64 DAS in C (``das_c.c``, threaded), for grids
                  where the NumPy restatement is too slow;
* ``scene``    -- the float64 forward model of moving point-scatterer scenes
                  (the reference's simulate_point pulse, src/rcabeam/sim.py:131-189).

Only the test suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import it, and only as the
checker or the timed CPU baseline.  The product path (``rcabeam_b200``) never
imports or calls anything here; it fails loudly when its CUDA library is
missing.

Parity pin: the oracle is checked against golden vectors generated by the
reference's own NumPy implementation (``tests/golden/make_golden.py``) and
against the reference test suite's known answers (``tests/test_oracle.py``).
"""
