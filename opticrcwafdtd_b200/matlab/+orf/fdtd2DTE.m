function out = fdtd2DTE(sim)
%FDTD2DTE orf.fdtd2DTE on the B200 engine: orf.fdtd2D with sim.pol = "TE"
%   (toolbox/+orf/fdtd2DTE.m:33-34).  See orf.fdtd2D in this folder.
out = orf_fdtd_mex('fdtd2DTE', mexsim(sim));
end
