"""FP64 CPU restatement of the PROFESS density-solve path (test infrastructure).

This package is the parity oracle for ``profess_b200``.  It is NOT part of the
product: only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg
of ``bench.py`` may import it, and only as the checker or the timed CPU
reference.  The product path never calls into it.

Each function restates one routine of EACcodes/PROFESS (Fortran 90) and cites
the reference file and line range it follows.  FFTs use ``scipy.fft`` with the
reference's convention: the real-to-complex forward transform is scaled by
1/N and the complex-to-real backward transform is unscaled
(``Source/Fourier_v1.f90:389-393``).  Arrays are indexed ``a[i1, i2, i3]`` with
x = i1; converting to the device layout (x fastest) is ``a.ravel(order="F")``.

Parity pinning: the reference Fortran cannot be compiled in this environment
(no Fortran compiler, no FFTW3), so the oracle is pinned against the golden
energy tables printed in the reference's own sample outputs
(``test/optIon/sampleoutput/displaced.out``, ``test/optDen/sample.output``);
see ``tests/test_oracle_golden.py``.
"""
