"""Run logs in the format of the reference (``pf_kks/runlog.py:15-140``).

``dtime.txt`` records the material state every 100 steps (every attempt of
such a step) and every rejected step; ``log.txt`` records the residual of every
adaptive decision. The GPU step emits one device record per line to write, in
program order, and the host formats them here; the strings are kept identical
to the reference's so that logs can be compared byte for byte.
"""

import os


def _e(x):
    return "{0:.2e}".format(x)


class RunLog:
    def __init__(self, directory, enabled=True):
        self.enabled = enabled
        self.log_path = os.path.join(directory, "log.txt")
        self.dtime_path = os.path.join(directory, "dtime.txt")
        self._log = []
        self._dtime = []
        if enabled:
            os.makedirs(directory, exist_ok=True)
            with open(self.log_path, "w") as f:
                f.write("start simulation\n")
            with open(self.dtime_path, "w") as f:
                f.write("print time steps\n")

    def flush(self):
        """Append the buffered lines to the files."""
        if not self.enabled:
            return
        if self._log:
            with open(self.log_path, "a") as f:
                f.write("".join(self._log))
            self._log.clear()
        if self._dtime:
            with open(self.dtime_path, "a") as f:
                f.write("".join(self._dtime))
            self._dtime.clear()

    def state(self, istep, T, D, L, Meta, Omega0, dtime_s):
        if self.enabled:
            self._dtime.append("step: " + str(istep) + ", T= " + "{0:.3f} ".format(T) + " D= " + _e(D) + " L= "
                               + _e(L) + " Meta= " + _e(Meta) + " Vm= " + _e(Omega0) + " dtime_s= "
                               + "{0:.2f}".format(dtime_s) + " \n")

    @staticmethod
    def _terms(res, sep):
        return ("Residual = " + _e(abs(res.total)) + "," + " Energy_deriv= " + _e(res.energy_derivative) + ","
                + " Potentiel_grad= " + _e(res.diffusion_term) + "," + " eta_term= " + _e(res.allen_cahn_term)
                + sep + " temp_term= " + _e(res.temperature_term))

    def rejected(self, istep, iteration, dtime_s, res, energy_s):
        if self.enabled:
            self._log.append("step " + str(istep) + ": RE>resmax\n" + self._terms(res, "") + ","
                             + "         Energy= " + _e(energy_s) + "\n")
            self._dtime.append("RE>resmax\n" + "repeat istep " + str(istep) + " : iteration " + str(iteration)
                               + " dtime_s:  " + _e(dtime_s) + "\n" + "\n")

    def accepted(self, istep, res, energy_s):
        if self.enabled:
            self._log.append("step: " + str(istep) + ", We get  (resmin <RE <resmax) ;  go to step " + str(istep + 1)
                             + "\n" + self._terms(res, ",") + "," + "         Energy= " + _e(energy_s) + "\n")

    def enlarged(self, istep, res, energy_s):
        if self.enabled:
            self._log.append(" We get  :RE <resmin;  go to step " + str(istep) + "\n" + self._terms(res, ",")
                             + "         Energy= " + _e(energy_s) + "\n")
