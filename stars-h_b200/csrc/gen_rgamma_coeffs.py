"""Prints the Taylor coefficients of 1/Gamma(1+z) about z = 0 that
kernel_entry.cuh embeds (kRGammaCoef), computed with mpmath at 50 digits.

    python gen_rgamma_coeffs.py
"""
import mpmath as mp

mp.mp.dps = 50
for c in mp.taylor(lambda z: mp.rgamma(1 + z), 0, 28):
    print(f"    {mp.nstr(c, 25)},")
