"""Material laws with the reference's interface (``snoopy/materials.py``).

The kernels read a material through the same duck-typed methods the reference's
Cython layer uses (``fem_c/interface_c.pyx:57-68, 226-234``): ``get_type_spec()``,
``get_spline_information()``, ``.value`` and ``evaluate_mu(0.0)``.

* ``Reluctance``: nu(|B|) as a PCHIP interpolant of (B, H/B) with nu[0] = nu[1]
  (``materials.py:298-311``), shipped to the kernels in piecewise-polynomial form
  ``(c[4, n_int], x[n_int + 1])`` (``materials.py:428-436``).
* ``ConstantReluctance``: type 0, ``value`` (``materials.py:486-536``).
* ``Permeability``: mu(log10 |H|) as an interpolating cubic B-spline (``splrep``),
  with H_min where the spline's slope vanishes in the first interval
  (``materials.py:30-62, 184-197``).
* ``ConstantPermeability``: type 0 (``materials.py:210-269``).
* ``Dilution``: the linear-in-z iron fraction of diluted steel (``materials.py:538-599``).

``atan_bh_table`` makes the B-H table of the saturating law
B(H) = mu0 H + Js (2/pi) atan(pi mu0 (mu_r - 1) H / (2 Js)); ``Reluctance.from_bh`` fits
it exactly like a table read from a material file.
"""

import json
import math

import numpy as np
from scipy.interpolate import PchipInterpolator, splev, splrep
from scipy.optimize import minimize_scalar

MU0 = 4e-7 * math.pi
NU0 = 1.0 / 4.0 / math.pi * 1e7  # vacuum reluctance, as ``fem_c/ctools.c:1230``


class Reluctance:
    """PCHIP reluctance nu(|B|) fitted to B-H data (``snoopy/materials.py:271-436``)."""

    def __init__(self, input_filename=None, B=None, H=None):
        if input_filename is not None:
            with open(input_filename) as f:
                mat_data = json.load(f)
            self.B_data = np.array(mat_data["BH_data"]["B(T)"], dtype=np.float64)
            self.H_data = np.array(mat_data["BH_data"]["H(A/m)"], dtype=np.float64)
        else:
            self.B_data = np.asarray(B, dtype=np.float64)
            self.H_data = np.asarray(H, dtype=np.float64)
        self.initialize_interpolation()

    @classmethod
    def from_bh(cls, B, H):
        return cls(B=B, H=H)

    def initialize_interpolation(self):
        # nu = H/B with nu[0] = nu[1]  (materials.py:305-308)
        self.nu = 0.0 * self.H_data
        self.nu[1:] = self.H_data[1:] / self.B_data[1:]
        self.nu[0] = self.nu[1]
        self.spl = PchipInterpolator(self.B_data, self.nu, extrapolate=True)

    def evaluate_nu(self, B_mag):
        return self.spl(B_mag)

    def evaluate_nu_derivative(self, B_mag):
        return self.spl.derivative()(B_mag)

    def get_type_spec(self):
        return 1

    def get_spline_information(self):
        """PP coefficients c[4, n_int] and breakpoints x[n_int + 1] (``materials.py:428-436``)."""
        return self.spl.c, self.spl.x


class ConstantReluctance:
    """Constant reluctance (``snoopy/materials.py:486-536``)."""

    def __init__(self, value):
        self.value = float(value)

    def evaluate_nu(self, B_mag):
        return self.value + 0.0 * np.asarray(B_mag)

    def evaluate_nu_derivative(self, B_mag):
        return 0.0 * np.asarray(B_mag)

    def get_type_spec(self):
        return 0


class Permeability:
    """B-spline permeability mu(x), x = log10 |H| (``snoopy/materials.py:8-208``)."""

    def __init__(self, input_filename=None, B=None, H=None):
        if input_filename is not None:
            import pandas as pd

            mat_data = pd.read_csv(input_filename)
            self.B_data = mat_data["B(T)"].values.astype(np.float64)
            self.H_data = mat_data["H(A/m)"].values.astype(np.float64)
        else:
            self.B_data = np.asarray(B, dtype=np.float64)
            self.H_data = np.asarray(H, dtype=np.float64)
        self.initialize_interpolation()

    @classmethod
    def from_bh(cls, B, H):
        return cls(B=B, H=H)

    def initialize_interpolation(self):
        # materials.py:38-62 (the report figure of the reference is not drawn)
        self.mu = np.zeros((len(self.H_data),))
        self.mu[1:] = self.B_data[1:] / self.H_data[1:]
        self.mu[0] = self.mu[1]
        self.x = np.zeros((len(self.H_data),))
        self.x[1:] = np.log10(self.H_data[1:])
        self.x[0] = 2 * self.x[1] - self.x[2]
        self.spl = splrep(self.x, self.mu)

        def obj_fcn(x):
            return abs(splev(x, self.spl, der=1))

        self.x_min = minimize_scalar(obj_fcn, bounds=[self.x[0], self.x[1]]).x
        self.H_min = 10.0 ** self.x_min

    def evaluate_mu(self, H_mag, relative=False):
        H = np.atleast_1d(np.asarray(H_mag, dtype=np.float64)).copy()
        H[H < self.H_min] = self.H_min
        mu = splev(np.log10(H), self.spl)
        return mu / 4 / np.pi * 1e7 if relative else mu

    def evaluate_mu_derivative(self, H_mag, relative=False):
        H = np.atleast_1d(np.asarray(H_mag, dtype=np.float64)).copy()
        H[H < self.H_min] = self.H_min
        d_mu = splev(np.log10(H), self.spl, der=1) / H / np.log(10)
        return d_mu / 4 / np.pi * 1e7 if relative else d_mu

    def get_spline_information(self):
        """Knots t, coefficients c, degree k, H_min and mu below H_min (``materials.py:184-197``)."""
        return self.spl[0], self.spl[1], self.spl[2], self.H_min, self.evaluate_mu(np.array([0.0]))[0]

    def get_type_spec(self):
        return 1


class ConstantPermeability:
    """Constant permeability (``snoopy/materials.py:210-269``)."""

    def __init__(self, mu):
        self.mu = float(mu)

    def evaluate_mu(self, H_mag, relative=False):
        v = self.mu / 4 / np.pi * 1e7 if relative else self.mu
        return v + 0.0 * np.asarray(H_mag, dtype=np.float64)

    def evaluate_mu_derivative(self, H_mag, relative=False):
        return 0.0 + 0.0 * np.asarray(H_mag, dtype=np.float64)

    def get_type_spec(self):
        return 0


class Dilution:
    """Diluted steel: the iron fills only part of a magnet's cross section, and the part
    changes linearly along z (``snoopy/materials.py:538-599``).

    Each of the four x boundaries (middle gap, core, void, yoke) runs on a straight line
    from x_1 at z = z_pos to x_2 at z = z_pos + z_len, x(z) = c + m z.  The dilution factor
    is a ratio of two widths, s(z) = (c_num + z m_num) / (c_den + z m_den): for magnet type 1
    (yoke - void) / (core - gap), for type 3 the inverse.  The curl-curl kernels evaluate s at
    every quadrature point and use nu = s PCHIP(s |B|), nu' = s^2 PCHIP'(s |B|)
    (``fem_c/ctools.c:1665-1680``).
    """

    def __init__(self, x_mgap_1, x_core_1, x_void_1, x_yoke_1, x_mgap_2, x_core_2, x_void_2, x_yoke_2, z_pos, z_len,
                 mag_type=1):
        def line(x1, x2):
            return (x1 * (z_len + z_pos) - x2 * z_pos) / z_len, (x2 - x1) / z_len

        c_gap, m_gap = line(x_mgap_1, x_mgap_2)
        c_core, m_core = line(x_core_1, x_core_2)
        c_void, m_void = line(x_void_1, x_void_2)
        c_yoke, m_yoke = line(x_yoke_1, x_yoke_2)
        outer = (c_yoke - c_void, m_yoke - m_void)
        inner = (c_core - c_gap, m_core - m_gap)
        if mag_type == 1:
            num, den = outer, inner
        elif mag_type == 3:
            num, den = inner, outer
        else:
            raise ValueError(f"magnet type {mag_type} unknown (1 or 3)")
        self.c_num, self.m_num = num
        self.c_den, self.m_den = den
        self.mag_type = mag_type

    def coefficients(self):
        """(c_num, m_num, c_den, m_den), the order the C interface takes them in."""
        return (float(self.c_num), float(self.m_num), float(self.c_den), float(self.m_den))

    def evaluate(self, z):
        """s(z), as ``eval_dilution`` (``fem_c/ctools.c:124-128``)."""
        z = np.asarray(z, dtype=np.float64)
        return (self.c_num + z * self.m_num) / (self.c_den + z * self.m_den)


def atan_bh(H, mu_r=3000.0, Js=1.9):
    """B(H) = mu0 H + Js (2/pi) atan(pi mu0 (mu_r - 1) H / (2 Js))."""
    H = np.asarray(H, dtype=np.float64)
    return MU0 * H + Js * (2.0 / math.pi) * np.arctan(math.pi * MU0 * (mu_r - 1.0) * H / (2.0 * Js))


def atan_h_of_b(B, mu_r=3000.0, Js=1.9):
    """Inverse of ``atan_bh`` by bisection (monotone law), to full float64 precision."""
    B = np.atleast_1d(np.asarray(B, dtype=np.float64))
    lo = np.zeros_like(B)
    hi = np.maximum(B / MU0, 1.0)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        below = atan_bh(mid, mu_r, Js) < B
        lo = np.where(below, mid, lo)
        hi = np.where(below, hi, mid)
    return 0.5 * (lo + hi)


def atan_bh_table(mu_r=3000.0, Js=1.9, n_knots=40, n_far=10, B_far=1e7):
    """B-H table of the atan law with ``n_knots`` B values.

    ``n_knots - n_far`` knots cover 0 .. 1.37 Js (uniform up to 0.8 Js, then denser through
    the knee); the last ``n_far`` are log-spaced from 1.58 Js to ``B_far``, where nu is
    within 1e-7 of nu0.  Like the reference's material files (which run to 1e4-1e7 T), this
    keeps the PCHIP's extrapolation beyond the last knot physical for any Newton iterate.
    """
    n_near = n_knots - n_far
    n_lin = n_near // 2
    b_lin = np.linspace(0.0, 0.8 * Js, n_lin, endpoint=False)
    b_knee = 0.8 * Js + (1.37 - 0.8) * Js * np.linspace(0.0, 1.0, n_near - n_lin) ** 1.3
    b_far = np.logspace(np.log10(1.58 * Js), np.log10(B_far), n_far)
    B = np.concatenate([b_lin, b_knee, b_far])
    H = atan_h_of_b(B, mu_r, Js)
    H[0] = 0.0
    return B, H


def atan_reluctance(mu_r=3000.0, Js=1.9, n_knots=40):
    """Iron reluctance of the saturating atan law, as a PCHIP ``Reluctance``."""
    B, H = atan_bh_table(mu_r, Js, n_knots)
    return Reluctance.from_bh(B, H)


def atan_permeability(mu_r=3000.0, Js=1.9, n_knots=40, H_max=1e7):
    """Permeability mu(log10 H) of the atan law, fitted like a B-H material file."""
    H = np.concatenate([[0.0], np.logspace(-1, math.log10(H_max), n_knots - 1)])
    B = atan_bh(H, mu_r, Js)
    return Permeability.from_bh(B, H)
