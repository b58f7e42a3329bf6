function build_mex()
%BUILD_MEX compile orf_fdtd_mex (the MATLAB gateway of liborf_fdtd.so) next to
%   this file.  Build the library first: python -m opticrcwafdtd_b200.build.
%   Then: addpath(fileparts(which('build_mex')), '-begin') and call
%   orf.fdtd2D / orf.fdtd2DTE / orf.fdtd3D as with the reference's toolbox.
here = fileparts(mfilename('fullpath'));
repo = fileparts(fileparts(here));
lib = fullfile(repo, 'opticrcwafdtd_b200', 'lib');
mex('-R2018a', ['-I' fullfile(repo, 'include')], fullfile(here, 'orf_fdtd_mex.c'), ['-L' lib], '-lorf_fdtd', ...
    ['LDFLAGS=$LDFLAGS -Wl,-rpath,' lib], '-outdir', here);
end
