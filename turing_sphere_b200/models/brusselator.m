% Brusselator kinetics on the unit sphere (stripes and spots).
%
%   u_t = D1 lap(u) + A - (B+1) u + u^2 v
%   v_t = D2 lap(v) + B u - u^2 v
%
% IMEX Euler as in schnakenberg.m: explicit reaction on the grid, implicit
% diffusion per coefficient.  Spectral arrays are 2 x nlm, grid arrays npts x 1.

function [U, V, u, v] = init(noise, A, B)
  U = analys(A + noise);
  V = analys((B / A) * ones(numel(noise), 1));
  u = synth(U);
  v = synth(V);
end

function [Un, Vn, u, v] = step(U, V, lam, A, B, D1, D2, dt)
  u = synth(U);
  v = synth(V);
  uuv = u .* u .* v;
  Un = (U + dt * analys(A - (B + 1) * u + uuv)) ./ (1 + (dt * D1) * lam);
  Vn = (V + dt * analys(B * u - uuv))           ./ (1 + (dt * D2) * lam);
end
