function out = fdtd3D(sim)
%FDTD3D orf.fdtd3D on the B200 engine: 3D Yee FDTD with CPML, TF/SF plane
%   source and planar DFT monitors.  out = orf.fdtd3D(sim) takes the sim
%   struct of toolbox/+orf/fdtd3D.m (fdtd3D.m:11-24; courant default
%   0.99/sqrt(3)) and returns out.flux, out.mon(q).Ea/Eb/Ha/Hb, converged,
%   steps, time, wallTime (fdtd3D.m:26-29), computed on the GPU through the
%   MEX gateway orf_fdtd_mex.  Reaching maxTime warns fdtd3D:notConverged.
%   Path set-up as for orf.fdtd2D in this folder.
out = orf_fdtd_mex('fdtd3D', mexsim(sim));
end
