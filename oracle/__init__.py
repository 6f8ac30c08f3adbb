"""CPU oracle for the Mobile V2 terrain step -- TEST INFRASTRUCTURE ONLY.

This package restates, in NumPy, the algorithms of the reference project
(wordxzl03-oss/Iron-soil-physical-simulation-algorithom-for-Isaac-Sim) that the
CUDA library replaces.  It is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may import
it.  The product path (the ``soilb200`` package and ``libsoilb200.so``) never
calls into this package and has no CPU fallback.

Pinning: every module here is checked against golden fixtures in
``tests/golden/`` that were produced by running the reference's own Python
implementation (``tests/golden/make_golden.py``) and against the JSON reports
the reference ships (``outputs/mobile_v2_reference/*.json``).

Modules
-------
mobile_v2     FP64 restatement of ``MobileV2ReferenceSolver`` (bit-level mirror).
fixed_point   CPU mirror of the 32-bit fixed-point/FP32 production arithmetic.
relax         ``relax_critical_slope`` and the device compact-frontier schedule.
labels        cohesive-yield initialisation and canonical union-find labels.
"""
