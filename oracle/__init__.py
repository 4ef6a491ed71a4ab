"""CPU oracle for the far-field ptychography hot path -- TEST INFRASTRUCTURE ONLY.

This package restates, in FP64 NumPy (and, for the timed CPU baseline, in
torch on the CPU), the reference algorithm of
zhixuanh0710/conventional-ptychography-reconstruction for the path that the
CUDA library replaces:

* ``forward_model``  -- scan geometry (utils/optics.py:68-99), the forward
  model (utils/optics.py:102-112, Recovery.py:288-292), the three losses
  (Recovery.py:294-305) and the adjoint that torch autograd computes for them
  (Recovery.py:316);
* ``inr``            -- the complex-exponential MLP (models/complex_inr.py:6-82),
  the multi-resolution hash encoding consumed through tiny-cuda-nn
  (models/complex_inr.py:130-145) restated from the published Instant-NGP
  method, Fourier upsampling (models/complex_inr.py:252-271) and Adam;
* ``torch_cpu_path`` -- the reference's own per-frame torch CPU loop
  (forward + inline loss + autograd), used as the timed CPU baseline.

Only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` may import this package, and only as
the checker or the CPU baseline.  The product path (the CUDA library and its
Python host code) never imports it and has no CPU fallback.

Parity pinning: the forward model, losses, adjoint, scan indices, probe
centring, Haar sparsity and ComplexMLP are pinned against golden vectors
produced by importing the reference itself (``tests/golden/make_golden.py``).
The HashGrid restatement has no reference output to pin against
(tiny-cuda-nn is an unpinned, absent third-party dependency): parity unpinned
for that component.
"""
