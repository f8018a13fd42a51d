% Build the three MATLAB gateways against libmcsart (sm_100a engine).
% Run from the repository root after `python -m mcsart_b200.build`.
inc = ['-I' fullfile(pwd, 'include')];
lib = ['-L' fullfile(pwd, 'mcsart_b200', 'lib')];
src = fullfile(pwd, 'mcsart_b200', 'mex');
mexcuda(inc, lib, '-lmcsart', fullfile(src, 'entry_AUMISART.cpp'), '-outdir', 'bin');
mexcuda(inc, lib, '-lmcsart', fullfile(src, 'mex_backprojection.cpp'), '-outdir', 'bin');
mexcuda(inc, lib, '-lmcsart', fullfile(src, 'mex_diff.cpp'), '-outdir', 'bin');
