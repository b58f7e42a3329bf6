function out = fdfd2D(x, z, epsr, lambda0, J, opts)
%FDFD2D orf.fdfd2D on the B200 engine: the 2D TE frequency-domain solver
%   with its adjoint.  out = orf.fdfd2D(x, z, epsr, lambda0, J) solves
%       (1/s_x) d/dx((1/s_x) dE/dx) + (1/s_z) d/dz((1/s_z) dE/dz) + k0^2 eps E = -J
%   for E = E_y on the grid x (nx), z (nz) (uniform, equal spacing) with
%   stretched-coordinate PML and E = 0 outside, as toolbox/+orf/fdfd2D.m
%   documents (options Npml, default [30 30], and PmlReflection, 1e-8).
%   The factors stay on the GPU while out (or a handle taken from it) lives:
%     out.E, out.k0
%     out.solve(J2)   E for another current, the same factors
%     out.adjoint(g)  lam with A.' lam = g: for c = sum(g .* E),
%                     dc/deps = -k0^2 lam .* E
%     out.fluxX(ix, iz) / out.fluxZ(iz, ix)  power through a vertical /
%                     horizontal line (> 0 toward +x / +z), centred differences
arguments
    x (:, 1) double
    z (:, 1) double
    epsr double
    lambda0 (1, 1) double
    J double
    opts.Npml (1, :) double = [30 30]
    opts.PmlReflection (1, 1) double = 1e-8
end
f = orf.FdfdFactors(orf_fdtd_mex('fdfd2D_factor', x, z, epsr, lambda0, opts.Npml, opts.PmlReflection));
d = x(2) - x(1);
k0 = 2 * pi / lambda0;
E = f.solve(J);
out.E = E;
out.k0 = k0;
out.solve = @(J2) f.solve(J2);
out.adjoint = @(g) f.adjoint(g);
out.fluxX = @(ix, iz) d / (2 * k0) * sum(imag(conj(E(ix, iz)) .* (E(ix + 1, iz) - E(ix - 1, iz)) / (2 * d)));
out.fluxZ = @(iz, ix) d / (2 * k0) * sum(imag(conj(E(ix, iz)) .* (E(ix, iz + 1) - E(ix, iz - 1)) / (2 * d)));
end
