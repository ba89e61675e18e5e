"""B200 k-mer association test (the 1-D column-mode test of SuperGWAS's kgwas).

The compute path is native: ``lib/libkgwas_cuda.so`` (sm_100a CUDA behind the
C ABI of ``include/kgwas_cuda.h``) and ``bin/kgwas`` (drop-in command line).
``supergwas_b200.api`` is a ctypes binding of that C ABI.
"""
__all__ = ["api", "build", "synth"]
