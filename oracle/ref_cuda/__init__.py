"""The reference's own CUDA kernels for the 128x128 SSB object, built and run
as a CHECKER and BASELINE (test infrastructure, never the product).

bobleesj/quantem.gpu 0.0.1rc6 keeps its CUDA as source strings inside Python
modules and JIT-compiles them with NVRTC through CuPy
(src/quantem/gpu/ssb/compute/cuda/kernels/common.py:620-622 assembles the
module, :708 gives the compile options). CuPy is not installed here, so
``build_ref.py`` reads those strings with ``ast`` from the reference tree
(``build_ref.reference_root()``, present only in the build container), assembles the
module exactly as ``build_cuda_code`` does, and compiles it with nvcc and the
reference's options into ``oracle/_ref/ssb_fft128.cubin`` (git-ignored; the
built file travels to the GPU box, the source does not).

``harness.py`` loads that cubin with cuda-python and replays
``SSBEngine._run_correction_pipeline`` + ``reconstruct_object``
(engine.py:934-971, 1109-1151) for B > 1024 BF pixels at 128x128 scans: the
pk element-wise kernel (engine.py:217-231, restated), then the reference's
``ifft128_rows_fused_pk_t32_mr8_packed`` and ``ifft128_cols_t32_mr8``
(fft128.py:26-150, 353-397) with the engine's grids (common.py:768-816), then
the mean over BF pixels. The reference's Fourier-sum kernel
(``ssb128_corrected_fourier_sum_t256``) is never launched: the reference
itself disables it above 1024 BF pixels because it faults there
(engine.py:1128-1134).
"""
