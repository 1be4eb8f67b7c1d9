"""Dimensionless normalisation of the 1D2V problem.

Mirrors ``Reference(triplet, mass_fraction)`` of crewsdw/Vlasov1D2V (``main/reference.py:13-63``):
the same attribute names and the same formulas, evaluated in the same order, so the
coefficients (acceleration multiplier, Poisson coefficient, thermal velocity, cyclotron and
plasma frequencies) are bit-identical to the reference's.  ``info_file`` writes the run
description file in the reference's line layout (``main/reference.py:66-141``), which
``ReadData`` parses by line number.
"""
import datetime

import numpy as np

# physical constants (SI)
me = 9.10938188e-31
mp = 1.67262158e-27
e = 1.60217646e-19
eps0 = 8.854187e-12
mu0 = 4.0e-7 * np.pi
c = 1.0 / np.sqrt(eps0 * mu0)


class Reference:
    def __init__(self, triplet, mass_fraction):
        self.n = triplet[0]
        self.T = triplet[1]
        self.TeTi = triplet[2]
        self.Ld = np.sqrt(eps0 * self.T * self.TeTi / (self.n * e))
        self.mass_fraction = mass_fraction
        self.p = e * self.n * self.T
        self.B = np.sqrt(self.p * mu0)
        self.vth = np.sqrt(e * self.T / mp)
        self.v = self.B / np.sqrt(mu0 * mp * self.n)
        self.tau = self.Ld / self.v
        self.omp_p_tau = self.tau * np.sqrt(e * e * self.n / (eps0 * mp))
        self.omp_e_tau = self.tau * np.sqrt(e * e * self.n / (eps0 * me * self.mass_fraction))
        self.omc_p_tau = self.tau * e * self.B / mp
        self.omc_e_tau = self.tau * e * self.B / (me * self.mass_fraction)
        self.dp = c * self.tau / self.omp_p_tau
        self.ze = -1.0
        self.zi = +1.0
        self.ae = self.mass_fraction * me / mp
        self.ai = +1.0
        self.Ti = self.T
        self.Te = self.TeTi * self.T
        self.vt_i = np.sqrt(e * self.Ti / mp) / self.v
        self.vt_e = np.sqrt(e * self.Te / (me * self.mass_fraction)) / self.v
        self.cs = np.sqrt(e * (self.Te + self.Ti) / mp) / self.v
        self.deb_norm = (self.vt_e * self.v) / (self.omp_e_tau / self.tau)
        self.length = self.deb_norm
        self.electron_acceleration_multiplier = (self.ze / self.ae) * (self.length / self.dp)
        self.ion_acceleration_multiplier = (self.zi / self.ai) * (self.length / self.dp)
        self.charge_density_multiplier = -self.omp_p_tau ** 2.0 * (self.dp / self.length)

    def info_file(self, info_name, geometry_info, time_info):
        """Write the run description (same line positions as the reference's file)."""
        g = geometry_info
        final_time, write_time, courant_number, order_t = time_info[:4]
        lines = [
            "######################################",
            "### V-high-order Run File ############",
            "######################################",
            "Run performed " + datetime.datetime.today().strftime("%Y-%m-%d"),
            "",
            "Basis Triplet:",
            "Ref density:                           " + "{:.2E}".format(self.n) + " [m^-3]",
            "Ref temperature:                       " + "{:.2E}".format(self.T) + " [eV]",
            "Ref length (Debye):                    " + "{:.2E}".format(self.length) + " [m]",
            "",
            "Values Inferred from Triplet:",
            "Ref velocity:                          " + "{:.2E}".format(self.v) + " [m/s]",
            "Ref time:                              " + "{:.2E}".format(self.tau) + " [s]",
            "Ref proton plasma frequency:           " + "{:.2E}".format(self.omp_p_tau / self.tau) + " [Hz]",
            "Ref electron plasma frequency:         " + "{:.2E}".format(self.omp_e_tau / self.tau) + " [Hz]",
            "Ref proton thermal velocity:           " + "{:.2E}".format(self.v) + " [m/s]",
            "Ref proton skin depth:                 " + "{:.2E}".format(self.dp) + " [m]",
            "",
            "Normalized Run Values (Dimensionless):",
            "Run density                            " + "{:.2f}".format(self.n / self.n),
            "Run omptau                             " + "{:.2f}".format(self.omp_p_tau),
            "Run proton thermal velocity            " + "{:.2f}".format(self.vt_i),
            "Run proton temperature                 " + "{:.2f}".format(self.Ti / self.T),
            "Run electron-ion temperature ratio     " + "{:.2f}".format(self.TeTi),
            "Run ometau                             " + "{:.2f}".format(self.omp_e_tau),
            "Run electron thermal velocity          " + "{:.2f}".format(self.vt_e),
            "Run electron temperature               " + "{:.2f}".format(self.Te / self.T),
            "Run Debye length                       " + "{:.2f}".format(self.Ld),
            "Run skin depth                         " + "{:.2f}".format(self.dp / self.length),
            "Electron acceleration coefficient      " + "{:.2E}".format(self.electron_acceleration_multiplier),
            "Proton acceleration coefficient        " + "{:.2E}".format(self.ion_acceleration_multiplier),
            "Poisson equation coefficient           " + "{:.2E}".format(self.charge_density_multiplier),
            "",
            "Grid and time-stepping parameters",
            "X elements:                    " + str(g[0, 2]),
            "U elements:                    " + str(g[1, 2]),
            "V elements:                    " + str(g[2, 2]),
            "X domain minimum:              " + "{:.2E}".format(g[0, 0]),
            "X domain maximum:              " + "{:.2E}".format(g[0, 1]),
            "Electron u-velocity minimum    " + "{:.2E}".format(g[1, 0]),
            "Electron u-velocity maximum    " + "{:.2E}".format(g[1, 1]),
            "Electron v-velocity minimum    " + "{:.2E}".format(g[2, 0]),
            "Electron v-velocity maximum    " + "{:.2E}".format(g[2, 1]),
            "Time to run:                   " + "{:.2f}".format(final_time),
            "Time per data write-out         " + "{:.2f}".format(write_time),
            "CFL number:                    " + "{:.2f}".format(courant_number),
            "Spatial element order:         " + str(g[0, 3]),
            "Velocity-u element order:      " + str(g[1, 3]),
            "Velocity-v element order:      " + str(g[2, 3]),
            "Temporal stepping order:       " + str(order_t),
        ]
        with open(info_name, "w") as fh:
            fh.write("\n".join(lines))
