function out = fdtd2D(sim)
%FDTD2D orf.fdtd2D on the B200 engine: 2D TE/TM Yee FDTD in the xz plane.
%   out = orf.fdtd2D(sim) takes the sim struct of the reference's
%   toolbox/+orf/fdtd2D.m (fields and defaults of fdtd2D.m:9-23 and
%   fdtd2DTE.m:7-25) and returns its out struct (fdtd2D.m:25-29: flux, fluxZ,
%   P, B, PZ, AZ, the TE aliases Ey, Hz, EyZ, HxZ or TM aliases Hy, Ez, HyZ,
%   ExZ, converged, steps, time, wallTime).  The time loop runs on the GPU in
%   liborf_fdtd.so, called through the MEX gateway orf_fdtd_mex; sim.useGPU
%   is accepted and ignored.  An error thrown by sim.progress stops the run
%   and is rethrown unchanged; reaching maxTime warns fdtd2D:notConverged.
%
%   Put the folder that holds this +orf (opticrcwafdtd_b200/matlab) on the
%   path ahead of the reference's toolbox/ (addpath(..., '-begin')): MATLAB
%   then finds these wrappers before the toolbox's P-code of the same names.
out = orf_fdtd_mex('fdtd2D', mexsim(sim));
end
