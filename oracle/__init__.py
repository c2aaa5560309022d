"""CPU oracle for the plasmonX per-frequency response solve.

TEST INFRASTRUCTURE ONLY.  Nothing in the ``plasmonx_b200`` package imports,
links or executes anything under ``oracle/``.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` use it, and only as the checker or as the timed CPU
restatement of the reference -- never as the thing measured for the GPU arm.

Contents
  keywords.py  minimal reader of the reference's keyword input file (the file
               the reference's Python front end writes and its Fortran reads,
               ``src/input_output/input_module.f90:156-258``)
  model.py     FP64 NumPy restatement of the wFQ / wFQFMu model: interaction
               tiles, Drude/Fermi conductance, right-hand sides, frequency
               diagonals, polarizability and cross sections
  gmres.py     restatement of the reference GMRES (``src/solvers/gmres_module.f90``)
  solve.py     the three solver modes per frequency
               (``src/solvers/algorithm_module.f90:189-630``)
  bem.py       DPCM/IEFPCM boundary-element restatement (``src/bem/bem_module.f90``)
  analysis.py  induced field and density at points, atomistic and BEM (the
               reference's analysis step, ``src/matrix/matrix_module.f90:1140-1464``)
  static.py    static FQ / FQFMu solves and the principal-axis rotation
               (``src/forcefield/fq_module.f90``, ``fqfmu_module.f90``)
  pairs.c      C (POSIX threads) restatement of the on-the-fly pair kernels
               (``src/matrix/matrix_module.f90:727-1125``), the timed CPU baseline

Parity pins: the oracle is checked against the numbers printed in the
reference's own regression logs and output files (``tests/*/reference/``) by
``tests/test_oracle_golden.py``, ``test_static_golden.py``,
``test_analysis_golden.py``, ``test_analysis_extra.py`` and
``test_outputs.py`` (77 of the reference's 83 regression tests); the
extracted fixtures live in ``tests/golden/`` together with the script that
extracted them.
"""
