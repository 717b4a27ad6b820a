"""CPU restatement of the reference rdcu solver -- TEST INFRASTRUCTURE ONLY.

This package is the parity oracle for the CUDA library in ``rdcu_b200``.  It restates,
in numpy/scipy, what the reference's CUDA C++ does on the hot path:

* ``problem``  -- coupling-term parsing, Y-index table, glibc ``rand()`` initial
  conditions and the binary file formats (reference ``rdcu.cu``).
* ``spectral`` -- the pseudospectral Y blocks and the dictionary RHS
  (reference ``rdcu.cu:78-106,117-184``).
* ``fd``       -- finite-difference stencils, FD Y blocks and the CSR Jacobian
  (reference ``rdcu.cu:108-149,186-250,385-596``).
* ``dp45``     -- the Dormand-Prince 4(5) stepper (reference ``dp45.cu``).
* ``bdf``      -- the variable-order NDF/BDF stepper (reference ``bdf.cu``), with a
  scipy sparse LU in place of cuDSS.
* ``gmres``    -- the restarted GMRES(40) that replaces cuDSS in the library, used to
  check on the CPU that its solves keep the stepper's decisions.
* ``run``      -- an emulation of the reference ``main``/``step_eval`` that writes the
  same output files (reference ``rdcu.cu:252-341,599-1273``).
* ``tangent``  -- the tangent-linear derivative of fixed-step DP45 on the oracle RHS,
  used to check the library's discrete adjoint by duality.
* ``lines``    -- defect-line extraction and frame correlation of 3D CGLE states
  (reference ``makelines.py``).
* ``cpu_port`` -- a faster host restatement of the pseudospectral RHS and DP45, timed
  as the CPU baseline of ``bench.py``.

Parity pinning: the oracle is checked against fixtures produced by the reference's
own nvcc build (``oracle/build_ref.sh``) under ``tests/golden``; see the generating
script there.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its ``cpu_baseline``
leg and its reference arm) may import this package, and only as the checker or the
timed CPU baseline -- never as a product code path.
"""
