% Allen-Cahn on the unit sphere: one species whose domains coarsen.
%
%   u_t = eps2 lap(u) + u - u^3
%
% IMEX Euler: explicit cubic reaction on the grid, implicit diffusion per
% spherical-harmonic coefficient.

function [U, u] = init(noise)
  U = analys(noise);
  u = synth(U);
end

function [Un, u] = step(U, lam, eps2, dt)
  u = synth(U);
  Un = (U + dt * analys(u - u.^3)) ./ (1 + (dt * eps2) * lam);
end
