"""dream_b200: DREAM's delay-and-sum beamformer on B200 (sm_100a).

Modules mirroring the reference call surface:
    dream_b200.das.das(...)      FP64, the reference ``das``
    dream_b200.das_f.das(...)    FP32, the reference ``das_f``
    dream_b200.beamformer.das_uni(...)   uniform grids
"""
__version__ = "0.1.0"
