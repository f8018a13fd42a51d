/* Empty stand-in for MATLAB's gpu/mxGPUArray.h (test infrastructure only). */
