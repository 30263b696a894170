"""CPU oracle for the single-sideband (SSB) ptychography hot path.

THIS PACKAGE IS TEST INFRASTRUCTURE. It is the checker, never the product:
only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` may import it. The product path (``quantem.gpu_b200``) never
imports, links or executes anything under ``oracle/`` and fails loudly when
its CUDA extension is missing.

Contents
--------
``ssb_oracle``
    FP64 numpy restatement of the reference SSB path
    (bobleesj/quantem.gpu ``src/quantem/gpu/ssb/compute/cuda/backend.py``,
    ``engine.py`` and ``kernels/common.py``): u64 mean diffraction pattern,
    bright-field selection, Hermitian scan FFT, probe geometry, the
    aberration-corrected "trotter" correction, object wave, phase and the
    phase-variance loss. The integer and selection steps reproduce the
    reference's float32 decisions exactly; the Fourier arithmetic is FP64.
``ssb_torch_spec``
    A CPU torch restatement of the reference's executable specification
    (``docs/kernels/ssb.md``), multi-threaded; the timed CPU baseline.

Parity pinning
--------------
The oracle is pinned against outputs of the reference itself, generated in
the development container by ``tests/golden/make_golden.py``: the reference's
own host code (``CudaSSBBackend._compute_bf_mask``, ``_extract_gqk``,
``__init__`` padding, ``SSBEngine.cache_rotation``) and its own vectorised
test restatement (``tests/test_ssb_cuda_128.py::_reference_phase_loss``) are
executed with numpy standing in for CuPy, and their outputs are committed as
fixtures under ``tests/golden/``. The reference's Swift known-answer test
(zero input, one BF pixel, dc = 1) and integer-sum checks are restated as
tests. The reference's GPU kernels themselves cannot run here (no CuPy, no
GPU), and cuFFT is replaced by FP64 pocketfft, so the FFT boundary is pinned
only to FP32 tolerance.
"""
