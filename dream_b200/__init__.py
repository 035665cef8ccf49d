"""dream_b200: DREAM's delay-and-sum beamformer on B200 (sm_100a).

Modules mirroring the reference call surface:
    dream_b200.das.das(...)                FP64, the reference ``das``
    dream_b200.das_f.das(...)              FP32, the reference ``das_f``
    dream_b200.beamformer.das_uni(...)     uniform grids
    dream_b200.beamformer.das_mixed(...)   FP32 / BF16 A-scan storage with the FP64 indices
    dream_b200.conv.fftconv_p(...)         column-wise convolution (A-scan synthesis),
    dream_b200.conv.conv_p(...)            the reference ``fftconv_p`` / ``conv_p``
    dream_b200.dreamrect.dreamrect(...)    spatial impulse response of a rectangular transducer
    dream_b200.dream_arr_rect.dream_arr_rect(...)  ... of an array of rectangular elements

Beyond the reference: dream_b200.autograd (adjoint, autograd, CG),
dream_b200.batch (many frames in one persistent launch), dream_b200.matrix
(the beamformer as a sparse matrix), dream_b200.parallel (frames and frame
splits over torch.distributed ranks).
"""
__version__ = "0.1.0"
