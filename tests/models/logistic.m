% Test model: logistic reaction f(u) = r u (1 - u).  From a uniform field the
% state stays uniform and diffusion (zero at l = 0) does nothing, so each step
% is the explicit Euler map of the scalar ODE.

function [U, u] = init(noise)
  U = analys(noise);
  u = synth(U);
end

function [Un, u] = step(U, lam, r, D, dt)
  u = synth(U);
  Un = (U + dt * analys(r * u .* (1 - u))) ./ (1 + (dt * D) * lam);
end
