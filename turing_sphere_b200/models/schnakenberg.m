% Schnakenberg kinetics on the unit sphere (spots).
%
%   u_t = D1 lap(u) + a - u + u^2 v
%   v_t = D2 lap(v) + b - u^2 v
%
% One IMEX Euler step: the reaction is evaluated on the grid and the diffusion
% solved implicitly per spherical-harmonic coefficient, where lap = -l(l+1).
% The caller provides synth/analys, lam = l(l+1) per coefficient, the seeded
% grid perturbation `noise` and the parameters.  Spectral arrays are 2 x nlm
% (real and imaginary rows), grid arrays npts x 1.  Both functions return the
% new spectral state, then the grid fields to show.

function [U, V, u, v] = init(noise, a, b)
  us = a + b;
  vs = b / (us * us);
  U = analys(us + noise);
  V = analys(vs * ones(numel(noise), 1));
  u = synth(U);
  v = synth(V);
end

function [Un, Vn, u, v] = step(U, V, lam, a, b, D1, D2, dt)
  u = synth(U);
  v = synth(V);
  uuv = u .* u .* v;
  Un = (U + dt * analys(a - u + uuv)) ./ (1 + (dt * D1) * lam);
  Vn = (V + dt * analys(b - uuv))     ./ (1 + (dt * D2) * lam);
end
