/* Empty stand-in for MATLAB's matrix.h (test infrastructure only). */
