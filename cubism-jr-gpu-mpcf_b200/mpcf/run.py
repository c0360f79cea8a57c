"""Simulation runner with the reference's command line.

    python -m mpcf.run -sim SodMPI -nx 128 -ny 8 -nz 8 -tend 0.2 -cfl 0.3 \\
        -nslices 8 -dumpinterval 0.05 -saveinterval 100 -fpath out

The reference picks the case with -sim (main.cpp:42-60).  Every case runs
the loop of Sim_SteadyStateMPI::run (Sim_SteadyStateMPI.cpp:183-229):

- dt_max = min(tend - t, tnextdump - t);
- one LSRK3 step with dt = min(cfl*h/sos, dt_max);
- a dump when (float)t == (float)tnextdump;
- a save every saveinterval steps;
- a stop after nsteps steps (0: no limit);
- a last dump at the end.

Set-up follows Sim_SteadyStateMPI::_setup (:26-70).  -tend, -cfl, -nslices,
-dumpinterval and -saveinterval are mandatory unless -dryrun.  -restart 1
continues from <fpath>/save.* (then dumps "restart_ic" and sets
tnextdump = fcount*dumpinterval).  Otherwise the case's initial condition is
set and dumped.

Flags keep the reference's names and defaults (its ArgumentParser's
"-key value" pairs), with these differences:

- The domain size, fixed at compile time in the reference (block sizes),
  is given at run time with -nx -ny -nz.
- -precision picks the arithmetic: fp32_ref (default, the reference's
  rounding), fp32, mixed or fp64.
- -autotune 1 (default) times the tile shapes first.
- -nslices is accepted and ignored: the state stays on the device.
- -SOSkernel is accepted; the sound speed is always the device reduction.
- One domain on one GPU: -npex, -npey, -npez must be 1 (linked z-slabs
  are `mpcf.decomp`).

Cases and their input files, read from the working directory as the
reference reads them:

- SteadyStateMPI: -rho -u -v -w -p -g -pc.
- SodMPI: -config x|y|z -reverse -x0 -rho1 -rho2 -u1 -u2 -p1 -p2 -g1 -g2
  -pc1 -pc2.
- 2DSBIMPI: -config (xy, xz, yx, yz, zx, zy) -reverse -mollfactor -x0
  -mach -rho -rhobubble -u -p -pbubble -g1 -g2 -pc1 -pc2.  Bubbles come from
  <config>bubbles.dat: a count, then "x y z r" per bubble
  (Sim_2DSBIMPI.cpp:120-154).
- SICCloudMPI: -rho0 -u0 -p0 -rhoB -uB -pB -pressureratio -shockNx/Ny/Nz
  -shockSx/Sy/Sz -g1 -g2 -pc1 -pc2.  Shapes come from cloud.dat: one
  "idx x y z r" line each (Sim_SICCloudMPI.h:148-173).
- StaticIC: -config (xy, ...) -fname: a running cell count in every field,
  dumped once; no steps and no run options.
"""
import os
import sys
import time

import numpy as np

from . import solver as S
from ._lib import PRECISIONS, MpcfError

CASES = ("SteadyStateMPI", "SodMPI", "2DSBIMPI", "SICCloudMPI", "StaticIC")
CASE_FLAGS = {
    "SteadyStateMPI": ("rho", "u", "v", "w", "p", "g", "pc"),
    "SodMPI": ("x0", "rho1", "rho2", "u1", "u2", "p1", "p2", "g1", "g2", "pc1", "pc2"),
    "2DSBIMPI": ("x0", "mach", "rho", "rhobubble", "u", "p", "pbubble", "g1", "g2", "pc1", "pc2"),
    "SICCloudMPI": ("rho0", "u0", "p0", "rhoB", "uB", "pB", "g1", "g2", "pc1", "pc2"),
}


class ArgumentError(Exception):
    pass


def _is_number(tok):
    try:
        float(tok)
        return True
    except ValueError:
        return False


class Arguments:
    """Options read like the reference's ArgumentParser
    (IO/ArgumentParser.h:102-127).  A token starting with "-" names an option.
    The tokens after it up to the next option are its value, joined by
    spaces, and an option with no value is "1".  A key given twice keeps its
    last value, and stray tokens are ignored.  A mandatory key that is
    missing is an error.  One difference: a negative number is a value here,
    where the reference would take it for an option name."""

    def __init__(self, argv):
        self.kv = {}
        key, vals = None, []
        for tok in list(argv) + ["-"]:
            if tok.startswith("-") and not _is_number(tok):
                if key is not None:
                    self.kv[key] = " ".join(vals) if vals else "1"
                key, vals = tok[1:], []
            elif key is not None:
                vals.append(tok)

    def has(self, key):
        return key in self.kv

    def str(self, key, default=None):
        if key in self.kv:
            return self.kv[key]
        if default is None:
            raise ArgumentError(f"mandatory argument -{key} is missing")
        return default

    def float(self, key, default=None):
        return float(self.str(key, None if default is None else repr(default)))

    def int(self, key, default=None):
        return int(self.str(key, None if default is None else str(default)))

    def bool(self, key, default=False):
        v = self.kv.get(key)
        if v is None:
            return default
        return v.lower() in ("1", "true", "yes", "on")


def _case_kwargs(args, case):
    kw = {k: args.float(k) for k in CASE_FLAGS[case] if args.has(k)}
    if case == "SodMPI":
        kw["config"] = args.str("config", "x")
        kw["reverse"] = int(args.bool("reverse"))
    elif case == "2DSBIMPI":
        kw["config"] = args.str("config")
        kw["reverse"] = int(args.bool("reverse"))
        kw["mollfactor"] = args.int("mollfactor", 1)
    return kw


def read_bubbles(path):
    """<config>bubbles.dat of 2DSBI: a count, then x y z r per bubble."""
    with open(path) as f:
        tok = f.read().split()
    if not tok:
        raise ArgumentError(f"{path} is empty")
    n = int(tok[0])
    vals = [float(x) for x in tok[1:1 + 4 * n]]
    if len(vals) != 4 * n:
        raise ArgumentError(f"{path}: {n} bubbles announced, {len(vals) // 4} found")
    return np.array(vals, np.float64).reshape(n, 4)


def read_cloud(path):
    """cloud.dat of the cloud collapse: "idx x y z r" per line."""
    rows = []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if len(tok) >= 5:
                rows.append([float(t) for t in tok[1:5]])
    return np.array(rows, np.float64).reshape(-1, 4)


def _sic_params(args):
    kw = {k: args.float(k) for k in CASE_FLAGS["SICCloudMPI"] if args.has(k)}
    if args.has("pressureratio"):
        kw["pressure_ratio"] = args.float("pressureratio")
    p = S.sic_params(**kw)
    for i, a in enumerate("xyz"):
        if args.has(f"shockN{a}"):
            p.shock_n[i] = args.float(f"shockN{a}")
        if args.has(f"shockS{a}"):
            p.shock_s[i] = args.float(f"shockS{a}")
    return p


class Simulation:
    """One case on one GPU, driven like the reference's Simulation::run."""

    def __init__(self, argv, out=sys.stdout):
        self.args = a = Arguments(argv)
        self.out = out
        self.case = a.str("sim", "SteadyStateMPI")
        if self.case not in CASES:
            raise ArgumentError(f"Unknown simulation case {self.case}")
        self.dryrun = a.bool("dryrun")
        if self.case == "StaticIC":
            # Sim_StaticIC::_setup parses no run options (Sim_StaticIC.cpp:61-71)
            self.config = a.str("config")
            if sorted(self.config) not in (sorted(c) for c in ("xy", "xz", "yz")) or len(self.config) != 2:
                raise ArgumentError(f"-config {self.config} is not possible")
            self.fname = a.str("fname", "staticIC")
        elif not self.dryrun:
            self.tend = a.float("tend")
            self.cfl = a.float("cfl")
            self.nslices = a.int("nslices")
            self.dumpinterval = a.float("dumpinterval")
            self.saveinterval = a.int("saveinterval")
            if not (self.cfl > 0 and self.dumpinterval > 0 and self.saveinterval >= 1):
                raise ArgumentError("-cfl and -dumpinterval must be positive, -saveinterval at least 1")
        self.verbosity = a.int("verb", 0)
        self.restart = a.bool("restart")
        self.nsteps = a.int("nsteps", 0)
        if any(a.int(k, 1) != 1 for k in ("npex", "npey", "npez")):
            raise ArgumentError("one domain on one GPU: -npex/-npey/-npez must be 1")
        self.dims = (a.int("nx"), a.int("ny"), a.int("nz"))
        self.precision = a.str("precision", "fp32_ref")
        if self.precision not in PRECISIONS:
            raise ArgumentError(f"-precision must be one of {', '.join(PRECISIONS)}")
        self.fpath = a.str("fpath", ".")
        self.autotune = a.bool("autotune", True)
        self.t, self.step, self.fcount = 0.0, 0, 0
        self.solver = None

    def log(self, msg):
        print(msg, file=self.out, flush=True)

    def _bc(self):
        if self.case == "SteadyStateMPI":
            return S.case_bc("steady")
        if self.case == "SodMPI":
            return S.case_bc("sod")
        if self.case == "SICCloudMPI":
            return S.case_bc("sic")
        return S.case_bc("sbi", self.args.str("config"))

    def _ic(self):
        s, case = self.solver, self.case
        if case == "SteadyStateMPI":
            s.ic_steady(**_case_kwargs(self.args, case))
        elif case == "SodMPI":
            s.ic_sod(**_case_kwargs(self.args, case))
        elif case == "2DSBIMPI":
            kw = _case_kwargs(self.args, case)
            s.ic_sbi(read_bubbles(f"{kw['config']}bubbles.dat"), **kw)
        else:
            if not os.path.exists("cloud.dat"):
                raise ArgumentError("Can not find cloud.dat")
            s.ic_sic_cloud(_sic_params(self.args), read_cloud("cloud.dat"))

    def _dump(self, basename="data"):
        name = "%s_%04d" % (basename, self.fcount)
        self.fcount += 1
        self.log("Dumping file %s at step %d, time %f" % (name, self.step, self.t))
        self.solver.dump(self.fpath, name, self.step)

    def _save(self):
        self.solver.save(self.fpath, self.t, self.step, self.fcount)

    def setup(self):
        os.makedirs(self.fpath, exist_ok=True)
        self.solver = S.Solver([self.dims], bc=[self._bc()], precision=self.precision)
        self.tnextdump = self.dumpinterval
        if self.restart:
            r = self.solver.restart(self.fpath)
            if r is None:
                raise ArgumentError("Loading restart file was not successful")
            self.t, self.step, self.fcount = r
            self.log("Restarting at step %d, physical time %f" % (self.step, self.t))
            self._dump("restart_ic")
            self.tnextdump = self.fcount * self.dumpinterval
        else:
            self._ic()
            self._dump()
        if self.autotune:
            best, ms = self.solver.autotune(reps=1)
            if self.verbosity:
                self.log("tiling %s: %.3f ms per stage" % (best, ms))

    def static_ic(self):
        """Sim_StaticIC (Sim_StaticIC.cpp:74-96): every field of every cell
        holds a running count, axis config[0] fastest, then config[1], then
        the third; dumped once as <fname>_0000."""
        n = dict(zip("xyz", self.dims))
        fast, mid = self.config
        slow = ({"x", "y", "z"} - {fast, mid}).pop()
        z, y, x = np.meshgrid(np.arange(n["z"]), np.arange(n["y"]), np.arange(n["x"]), indexing="ij")
        i = {"x": x, "y": y, "z": z}
        cnt = i[fast] + n[fast] * (i[mid] + n[mid] * i[slow])
        os.makedirs(self.fpath, exist_ok=True)
        self.solver = S.Solver([self.dims], bc=[S.case_bc("sod")], precision=self.precision)
        field = cnt.astype(self.solver.dtype).ravel()
        self.solver.set_state([field] * 7)
        self._dump(self.fname)

    def run(self):
        if self.case == "StaticIC":
            self.static_ic()
            return
        if self.dryrun:
            # the reference sets up its host grid and allocates no GPU; here
            # the solver is the GPU, so a dry run only checks the arguments
            self.log("Dry Run...")
            return
        self.setup()
        while self.t < self.tend:
            dt_max = min(self.tend - self.t, self.tnextdump - self.t)
            t0 = time.perf_counter()
            dt = self.solver.step(cfl=self.cfl, dt_max=dt_max)[0]
            if self.verbosity:
                # the reference times the sound speed and each stage under
                # -verb (LSRK3_IntegratorMPI.cpp:35-59); here one call runs them
                self.log("step time %.3f ms (sound speed, dt and three stages)" % ((time.perf_counter() - t0) * 1e3))
            self.t += dt
            self.step += 1
            err = self.solver.error_word()
            if err:
                raise MpcfError(-1, "device error word 0x%x after step %d" % (err, self.step))
            self.log("step id is %d, physical time %f (dt = %f)" % (self.step, self.t, dt))
            if np.float32(self.t) == np.float32(self.tnextdump):
                self.tnextdump += self.dumpinterval
                self._dump()
            if self.step % self.saveinterval == 0:
                self.log("Saving time step...")
                self._save()
            if self.step == self.nsteps:
                break
        self._dump()

    def close(self):
        if self.solver is not None:
            self.solver.close()
            self.solver = None


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    print(" ".join(["mpcf.run"] + list(argv)), flush=True)
    try:
        sim = Simulation(argv)
    except (ArgumentError, ValueError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    t0 = time.perf_counter()
    try:
        sim.run()
    except (ArgumentError, MpcfError, OSError) as e:
        print(f"Error: {e}", file=sys.stderr)
        return 1
    finally:
        sim.close()
    print("Walltime: %f" % (time.perf_counter() - t0), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
