"""CPU oracle for Rayleigh's per-timestep transform + implicit-solve path.

TEST INFRASTRUCTURE ONLY.  This package is a plain NumPy / SciPy restatement
of the reference algorithm (geodynamics/Rayleigh 1.2.0, Fortran).  It is used
by ``tests/`` as the parity checker, by ``__graft_entry__.smoke()`` as the
checker of one small GPU step, and by ``bench.py`` for the ``cpu_baseline``
leg and the ``--impl reference`` arm.  Nothing in ``rayleigh_b200`` imports it,
and the product path never calls it.

Parity pinning: the Legendre tables and transforms are pinned against the
reference's own NumPy port (``post_processing/spectral_utils.py``) through the
committed fixtures in ``tests/golden/`` (made by ``tests/golden/make_golden.py``)
and against the analytic known answers of ``src/Test_Suite/Test_SHT.F90``.
The full time step is pinned by the reference's own regression report of its
accuracy benchmark (``tests/c2001_case0/Benchmark_Reports/00000400``, taken
into ``tests/golden/c2001_case0.json`` by ``tests/golden/make_c2001.py``); the
Fortran reference itself cannot be compiled here (no Fortran compiler, MPI,
FFTW or LAPACK in the image).
"""
from .rayleigh_oracle import *  # noqa: F401,F403
