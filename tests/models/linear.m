% Test model: linear reaction f(u) = c u.  Each coefficient then follows
%   U <- U (1 + dt c) / (1 + dt D l(l+1))
% exactly, so a run can be checked against arithmetic.

function [U, u] = init(noise)
  U = analys(noise);
  u = synth(U);
end

function [Un, u] = step(U, lam, c, D, dt)
  u = synth(U);
  Un = (U + dt * analys(c * u)) ./ (1 + (dt * D) * lam);
end
