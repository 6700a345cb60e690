"""CPU oracle of the colour-class Metropolis sweep — TEST INFRASTRUCTURE, NOT PRODUCT CODE.

Only tests/, `__graft_entry__.smoke()` and `bench.py` (its CPU-baseline leg and its `--impl reference` arm)
may import, call, link or execute anything here, and only as the checker or as the timed CPU baseline.
The product (`spin_colour_kernel_b200`) never imports this package and has no CPU fallback.

Contents:
  philox.py   Philox4x32-10 and the uniform conversion of Triton's tl.randint4x / tl.rand4x (NumPy).
  sweep.py    The generated class kernel's arithmetic restated per class, vectorised in NumPy float32
              (generator.py:150-319): plain int8 / float32 chains, packed storage, sync control.
  bitwise.py  The bitwise multi-spin-coded Ising chain, shared and independent draws (bitwise.py:79-246).
  observables.py  FP64 energy, local field and magnetization (sampler.py:296-345).
  cpu_sweep.c The same sweep in C with OpenMP over replicas: the timed CPU baseline for the large
              workloads (build recipe: oracle/build.py).

Parity is pinned: tests/golden/*.npz were generated by running the reference itself (its CPU path, the
Triton interpreter) with tests/golden/make_golden.py, and tests/test_oracle.py checks this oracle against
every one of them.
"""
