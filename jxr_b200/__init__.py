"""B200-native JPEG XR reconstruction engine (sm_100a).

A drop-in for the GPU reconstruction path of the frames-sg/jxr decoder: the
C ABI of include/jxr_b200.h, bound here by `jxr_b200.api`.
"""
from .api import (ALPHA, COLOR, CONTENT, DEPTH, LAYOUT, STORE, Arena, CudaDecodePlan, CudaDecoderSession,
                  CudaError, CudaSubmission, Geometry, OutputFormat, Request, ResidentImage, ResidentSet, SynthImage, lib,
                  synth)

__all__ = ["ALPHA", "COLOR", "CONTENT", "DEPTH", "LAYOUT", "STORE", "Arena", "CudaDecodePlan",
           "CudaDecoderSession", "CudaError", "CudaSubmission", "Geometry", "OutputFormat", "Request", "ResidentImage",
           "ResidentSet",
           "SynthImage", "lib", "synth"]
