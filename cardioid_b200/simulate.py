"""Runs a Cardioid object.data deck on the fused engine: the caller side of
the hot path, as the reference's set-up (elec/initializeSimulate.cc) and
omp time loop (elec/simulationLoop.cc:150-243) use it.

    sim = simulate.load(["object.data", "tt06.fit.data"])
    out = sim.run(precision="fp64")          # maxLoop steps
    out["vm"], out["activation"], out["minmax"], out["print"]

    python -m cardioid_b200.simulate object.data tt06.fit.data --precision mixed --out run.npz

What a deck may hold, per class (keys and defaults as the reference reads
them):
  SIMULATE     anatomy, diffusion, reaction (list), stimulus (list), sensor
               (list), dt, maxLoop, loop, printRate, printGid,
               checkpointRate, checkpointType (binary | ascii) and, as a
               restart file merges them in, stateFile (loop and time from
               its header)
  ANATOMY      method = brick (cellType, dx dy dz, xSize ySize zSize or nx
               ny nz; elec/initializeAnatomy.cc:147-239) or pio (fileName;
               cardioid_b200.anatomy.read_anatomy), conductivity
  CONDUCTIVITY method = uniform (sigma11 sigma22 sigma33 sigma12 sigma13
               sigma23) or fibre (sigmaLi, sigmaTi: read with the pio
               anatomy's angles)
  DIFFUSION    method = FGR (any variant) or b200 (the fused engine),
               cuda (the 6-face rule: the split loop on the drop-in plugins),
               null (no diffusion); diffusionScale
  REACTION     method = BetterTT06 (cardioid_b200.tt06.params_from_object),
               cellTypes; SINGLECELL objects named by a reaction set its
               cells' initial state
  STIMULUS     method = box (xMin..zMax, elec/stimulusFactory.cc:96-110) or
               point (cell: a local cell index), pulse = periodic (vStim,
               tStart, duration, period, t0, tf)
  SENSOR       method = activationTime (its times come back from run() and
               go to out_dir/snapshot.<last loop>/<filename>#000000 in the
               reference's record format; the engine evaluates every step)
               or minMax (time, min, max, max - min every printRate steps
               to out_dir/dirname/filename, as MinMaxSensor::print)
Other methods raise ValueError (no silent substitution).
"""
import argparse
import os

import numpy as np

from . import anatomy as anatomy_mod
from . import objectdb, tissue, tt06


class Simulation:
    """A deck turned into engine inputs: tissue, reaction parameters and
    per-cell reaction ids, initial states, dt and step count."""

    def __init__(self, t, params, reaction_of_cell, states, dt, steps, sensors, print_rate, print_gid,
                 checkpoint_rate=0, checkpoint_binary=True, state_file=None, name="simulate",
                 diffusion_method="FGR"):
        self.diffusion_method = diffusion_method
        self.activation_file = None           # the activationTime SENSOR's file name, written at the end
        self.minmax_out = None                # the minMax SENSOR's (printRate, dirname/filename)
        self.checkpoint_rate = checkpoint_rate
        self.checkpoint_binary = checkpoint_binary
        self.state_file = state_file          # a restart's pio state file (loop and time from its header)
        self.name = name
        self.tissue = t
        self.params = params
        self.reaction_of_cell = reaction_of_cell
        self.states = states                  # None, or 18 x n initial states
        self.dt = dt
        self.steps = steps
        self.sensors = sensors
        self.print_rate = print_rate
        self.print_gid = print_gid

    def run(self, precision="fp64", steps=None, device=0, out_dir="."):
        """Runs the deck's steps (or `steps`) on the fused engine and returns
        Vm, activation times, min/max Vm and the printed rows (loop, time,
        gid, Vm whenever the loop count is a multiple of printRate, as the
        reference's printData).  A restart (stateFile) starts from that
        checkpoint's state, loop and time; with checkpointRate, checkpoints
        go to out_dir/snapshot.<loop> at every multiple of it (the
        reference's writeCheckpoint)."""
        from . import checkpoint, engine, sensors
        steps = self.steps if steps is None else int(steps)
        t = self.tissue
        if self.diffusion_method == "cuda":
            return self._run_split(precision, steps, device, out_dir)
        with engine.Engine(self.dt, precision=precision, device=device) as e:
            rid = [e.add_reaction(p) for p in self.params]
            tid = e.add_tissue(t, np.asarray(rid, np.uint8)[self.reaction_of_cell])
            if self.states is not None:
                for k in range(tt06.NSTATE):
                    e.write_state(tid, k, self.states[k])
            if self.state_file:
                checkpoint.restore(e, tid, t, self.state_file)
            rows, saved, mm_rows = [], [], []
            pos = int(np.searchsorted(t.gid, self.print_gid)) if self.print_rate else None
            loop0 = e.time(tid)[0]
            done = 0
            while done < steps:
                loop = loop0 + done
                k = steps - done
                mm_rate = self.minmax_out[0] if self.minmax_out else 0
                for rate in (self.print_rate, self.checkpoint_rate, mm_rate):
                    if rate:
                        k = min(k, rate - loop % rate)
                e.step(k)
                done += k
                loop = loop0 + done
                if self.print_rate and loop % self.print_rate == 0:
                    s, time = e.time(tid)
                    rows.append((s, time, self.print_gid, e.read_vm(tid)[pos]))
                if mm_rate and loop % mm_rate == 0:
                    lo, hi = e.minmax(tid)
                    mm_rows.append((e.time(tid)[1], lo, hi))
                if self.checkpoint_rate and loop % self.checkpoint_rate == 0:
                    saved.append(checkpoint.save(e, tid, t, binary=self.checkpoint_binary, name=self.name,
                                                 root=out_dir))
            e.sync()
            out = {"vm": e.read_vm(tid), "steps": done, "loop": e.time(tid)[0], "time": e.time(tid)[1],
                   "print": np.array(rows), "checkpoints": saved}
            if "activationTime" in self.sensors:
                out["activation"] = e.read_activation(tid)
                if self.activation_file:
                    loop, time = e.time(tid)
                    out["activation_file"] = sensors.write_activation(
                        os.path.join(out_dir, "snapshot.%012d" % loop), t.gid, out["activation"], loop, time,
                        (t.nx, t.ny, t.nz), (t.dx, t.dy, t.dz), filename=self.activation_file)
            if "minMax" in self.sensors:
                out["minmax"] = e.minmax(tid)
                if self.minmax_out:
                    out["minmax_file"] = sensors.write_minmax(os.path.join(out_dir, self.minmax_out[1]), mm_rows)
            return out


    def _run_split(self, precision, steps, device, out_dir="."):
        """The reference's omp loop on the drop-in plugins, for decks whose
        DIFFUSION is the 6-face "cuda" rule (CUDADiffusion): iStim from the
        stimuli in list order, one BetterTT06 plugin per reaction on its
        cells, the 6-face diffusion, Vm += dt (dVmR + dVmD + iStim), time +=
        dt, the activation rule after each step (elec/simulationLoop.cc:183-231)."""
        import torch
        from . import plugins, sensors
        if self.state_file or self.checkpoint_rate:
            raise ValueError("checkpoints and restarts run on the fused engine (FGR diffusion)")
        t = self.tissue
        dev = "cuda:%d" % device
        vm = torch.from_numpy(np.ascontiguousarray(t.vm0, dtype=np.float64)).to(dev)
        dvr, dvd, ist = torch.zeros_like(vm), torch.zeros_like(vm), torch.zeros_like(vm)
        act = torch.full_like(vm, -1.0)
        idx, rx = [], []
        for r, p in enumerate(self.params):
            cells = np.flatnonzero(self.reaction_of_cell == r).astype(np.int32)
            idx.append(torch.from_numpy(cells).to(dev))
            rx.append(plugins.BetterTT06(p, len(cells), self.dt, precision=precision, device=device))
            if self.states is not None and len(cells):
                for k in range(tt06.NSTATE):
                    rx[-1].setValues(k, self.states[k][cells])
        diff = plugins.CUDADiffusion(t, t.diffusion_scale, device=device) if t.diffusion_scale else None
        x, y, z = t.tuples()
        masks = []
        for st in t.stimuli:
            if st.mode == 1:
                m = t.gid == st.cell
            else:
                m = (x > st.xMin) & (x < st.xMax) & (y > st.yMin) & (y < st.yMax) & (z > st.zMin) & (z < st.zMax)
            masks.append(torch.from_numpy(m).to(dev))
        pos = int(np.searchsorted(t.gid, self.print_gid)) if self.print_rate else None
        rows, mm_rows, time = [], [], 0.0
        mm_rate = self.minmax_out[0] if self.minmax_out else 0
        for s in range(1, steps + 1):
            ist.zero_()
            for st, m in zip(t.stimuli, masks):
                v = st.value(time)
                if v != 0.0:
                    if st.mode == 1:
                        ist[m] += v
                    else:
                        ist[m] = v
            for r in range(len(rx)):
                if rx[r].nCells:
                    rx[r].calc(self.dt, idx[r], vm, ist, dvr)
            if diff is not None:
                diff.updateLocalVoltage(vm)
                diff.calc(dvd)
            vm.add_(self.dt * (dvr + dvd + ist))
            time += self.dt
            act = torch.where((act < 0) & (vm > 0), torch.full_like(act, time), act)
            if self.print_rate and s % self.print_rate == 0:
                rows.append((s, time, self.print_gid, float(vm[pos])))
            if mm_rate and s % mm_rate == 0:
                mm_rows.append((time, float(vm.min()), float(vm.max())))
        torch.cuda.synchronize(device)
        v = vm.cpu().numpy()
        out = {"vm": v, "steps": steps, "loop": steps, "time": time, "print": np.array(rows), "checkpoints": []}
        if "activationTime" in self.sensors:
            out["activation"] = act.cpu().numpy()
            if self.activation_file:
                out["activation_file"] = sensors.write_activation(
                    os.path.join(out_dir, "snapshot.%012d" % steps), t.gid, out["activation"], steps, time,
                    (t.nx, t.ny, t.nz), (t.dx, t.dy, t.dz), filename=self.activation_file)
        if "minMax" in self.sensors:
            out["minmax"] = (float(v.min()), float(v.max()))
            if self.minmax_out:
                out["minmax_file"] = sensors.write_minmax(os.path.join(out_dir, self.minmax_out[1]), mm_rows)
        return out


def _brick(obj):
    dx = objectdb.get_float(obj, "dx", 0.2)
    dy = objectdb.get_float(obj, "dy", 0.2)
    dz = objectdb.get_float(obj, "dz", 0.2)
    if any(k in obj for k in ("nx", "ny", "nz")):
        nx = int(objectdb.get_float(obj, "nx", 16))
        ny = int(objectdb.get_float(obj, "ny", 16))
        nz = int(objectdb.get_float(obj, "nz", 14))
    else:
        nx = int(objectdb.get_float(obj, "xSize", 3) / dx)
        ny = int(objectdb.get_float(obj, "ySize", 7) / dy)
        nz = int(objectdb.get_float(obj, "zSize", 20) / dz)
    cell = objectdb.get_str(obj, "cellType", "102")
    if cell == "random":
        raise ValueError("ANATOMY brick with cellType = random is not supported")
    n = nx * ny * nz
    return (nx, ny, nz), (dx, dy, dz), np.arange(n, dtype=np.int64), np.full(n, int(cell), np.int32)


def _uniform_sigma(obj, n):
    g = lambda k: objectdb.get_float(obj, k, 0.0)
    row = [g("sigma11"), g("sigma12"), g("sigma13"), g("sigma22"), g("sigma23"), g("sigma33")]
    return np.tile(np.array(row, dtype=np.float64), (n, 1))


def _stimulus(db, name, t):
    obj = db.find(name, "STIMULUS")
    method = objectdb.get_str(obj, "method", "undefined")
    pulse = objectdb.get_str(obj, "pulse", "periodic")
    if pulse != "periodic":
        raise ValueError("STIMULUS %s: pulse %s is not supported (periodic only)" % (name, pulse))
    g = lambda k, d: objectdb.get_float(obj, k, d)
    kw = dict(vStim=g("vStim", -52.0), tStart=g("tStart", 0.0), duration=g("duration", 1.0),
              period=g("period", 1000.0), t0=g("t0", -1000.0), tf=g("tf", 1e30))
    if method == "box":
        return tissue.BoxStim(xMin=g("xMin", -1), xMax=g("xMax", t.nx), yMin=g("yMin", -1), yMax=g("yMax", t.ny),
                              zMin=g("zMin", -1), zMax=g("zMax", t.nz), **kw)
    if method == "point":
        cell = int(g("cell", 0))
        return tissue.point_stim(int(t.gid[cell]), t.nx, t.ny, **kw)
    raise ValueError("STIMULUS %s: method %s is not supported (box, point)" % (name, method))


def load(paths, simulate=None, generate=None):
    """Compiles the deck files (in order, as the reference's object files)
    and builds the Simulation of the SIMULATE object `simulate` (the first
    one when not named).  A pio anatomy's file name is taken relative to the
    first deck file's directory."""
    paths = [paths] if isinstance(paths, str) else list(paths)
    db = objectdb.ObjectDB()
    for p in paths:
        db.compile_file(p)
    base = os.path.dirname(os.path.abspath(paths[0]))
    names = db.names("SIMULATE")
    if not names:
        raise ValueError("no SIMULATE object in the deck")
    sim = db.find(simulate or names[0], "SIMULATE")
    dt = objectdb.get_float(sim, "dt", 0.01)
    steps = int(objectdb.get_float(sim, "maxLoop", 0)) - int(objectdb.get_float(sim, "loop", 0))

    an = db.find(objectdb.get_str(sim, "anatomy", "anatomy"), "ANATOMY")
    amethod = objectdb.get_str(an, "method", "pio")
    cname = objectdb.get_str(an, "conductivity", "conductivity")
    cond = db.find(cname, "CONDUCTIVITY") if db.exists(cname, "CONDUCTIVITY") else {}
    cmethod = objectdb.get_str(cond, "method", "uniform") if cond else "pio"
    if amethod == "brick":
        grid, spacing, gid, ct = _brick(an)
        if cmethod != "uniform":
            raise ValueError("a brick anatomy takes a uniform CONDUCTIVITY")
        sigma = _uniform_sigma(cond, len(gid))
        t = tissue.Tissue(*grid, *spacing, gid, ct, sigma, np.full(len(gid), -83.0), [])
    elif amethod == "pio":
        fname = objectdb.get_str(an, "fileName", "snapshot.initial/anatomy#")
        kw = dict(dx=objectdb.get_float(an, "dx", 0.2), dy=objectdb.get_float(an, "dy", 0.2),
                  dz=objectdb.get_float(an, "dz", 0.2))
        if cmethod == "fibre":
            kw.update(conductivity="fibre", sigma_l=objectdb.get_float(cond, "sigmaLi", 0.3e-3),
                      sigma_t=objectdb.get_float(cond, "sigmaTi", 0.0315e-3))
        elif cmethod == "uniform":
            kw.update(conductivity="uniform")
        elif cmethod == "JHU":
            kw.update(conductivity="JHU", sigma_l=objectdb.get_float(cond, "sigmaLi", 0.3e-3),
                      sigma_t=objectdb.get_float(cond, "sigmaTi", 0.0315e-3),
                      jhu=dict(sheet_angle=objectdb.get_float(cond, "sheetAngle", 45.0),
                               rotation_matrix=int(objectdb.get_float(cond, "rotatationMatrix", 1)),
                               homogeneous_fiber=bool(objectdb.get_float(cond, "homogeneousFiber", 0))))
        t = anatomy_mod.read_anatomy(os.path.join(base, fname), **kw)
        if cmethod == "uniform":
            t.sigma = _uniform_sigma(cond, t.n)
    else:
        raise ValueError("ANATOMY method %s is not supported (brick, pio)" % amethod)

    dname = objectdb.get_str(sim, "diffusion", "diffusion")
    dobj = db.find(dname, "DIFFUSION") if db.exists(dname, "DIFFUSION") else {}
    dmethod = objectdb.get_str(dobj, "method", "FGR")
    if dmethod == "null":
        t.diffusion_scale = 0.0
    elif dmethod in ("FGR", "b200", "cuda"):
        t.diffusion_scale = objectdb.get_float(dobj, "diffusionScale", 1.0)
    else:
        raise ValueError("DIFFUSION method %s is not supported (FGR, b200, cuda, null)" % dmethod)

    rnames = objectdb.get_list(sim, "reaction")
    params, type_of, vm_init, states = [], {}, [], []
    have_states = False
    for r, rn in enumerate(rnames):
        robj = db.find(rn, "REACTION")
        if objectdb.get_str(robj, "method", "") != "BetterTT06":
            raise ValueError("REACTION %s: only BetterTT06 runs on the engine" % rn)
        params.append(tt06.params_from_object(db, rn, dt, generate=generate))
        for ct in objectdb.get_list(robj, "cellTypes"):
            if int(ct) in type_of:
                raise ValueError("duplicate cellTypes within the reaction models")
            type_of[int(ct)] = r
        v, st = tt06.initial_state_from_object(db, rn)
        have_states = have_states or bool(st)
        vm_init.append(v)
        states.append(st)
    missing = set(np.unique(t.cell_type).tolist()) - set(type_of)
    if missing:
        raise ValueError("no reaction for cellTypes %s" % sorted(missing))
    rx = np.array([type_of[int(c)] for c in t.cell_type], dtype=np.uint8)
    vm0 = np.array([v if v is not None else tt06.INITIAL_VM for v in vm_init])[rx]
    t.vm0 = vm0
    st_all = None
    if have_states:
        st_all = np.empty((tt06.NSTATE, t.n))
        for r in range(len(params)):
            sel = rx == r
            for k, name in enumerate(tt06.STATE_NAMES):
                st_all[k, sel] = states[r].get(name, tt06.INITIAL_STATE[name])

    t.stimuli = [_stimulus(db, s, t) for s in objectdb.get_list(sim, "stimulus")]
    sensor_objs = [db.find(s, "SENSOR") for s in objectdb.get_list(sim, "sensor") if db.exists(s, "SENSOR")]
    sensors = [objectdb.get_str(o, "method", "") for o in sensor_objs]
    act_file, minmax_out = None, None
    for o in sensor_objs:
        if objectdb.get_str(o, "method", "") == "activationTime":
            act_file = objectdb.get_str(o, "filename", "activationTime")
        if objectdb.get_str(o, "method", "") == "minMax":
            minmax_out = (int(objectdb.get_float(o, "printRate", 1)),
                          os.path.join(objectdb.get_str(o, "dirname", "sensorData"),
                                       objectdb.get_str(o, "filename", "minmax")))
    print_rate = int(objectdb.get_float(sim, "printRate", 0))
    print_gid = int(objectdb.get_float(sim, "printGid", float(t.gid[0])))
    state_file = objectdb.get_str(sim, "stateFile")
    if state_file:
        state_file = state_file if os.path.isabs(state_file) else os.path.join(base, state_file)
    out = Simulation(t, params, rx, st_all, dt, steps, sensors, print_rate, print_gid,
                      checkpoint_rate=int(objectdb.get_float(sim, "checkpointRate", 0)),
                      checkpoint_binary=objectdb.get_str(sim, "checkpointType", "binary") != "ascii",
                      state_file=state_file, name=simulate or names[0],
                      diffusion_method="cuda" if dmethod == "cuda" else "FGR")
    out.activation_file = act_file
    out.minmax_out = minmax_out
    return out


def main(argv=None):
    ap = argparse.ArgumentParser(description="Runs a Cardioid object.data deck on the B200 engine.")
    ap.add_argument("files", nargs="+", help="object files, in the order the reference would read them")
    ap.add_argument("--simulate", default=None, help="the SIMULATE object (default: the first)")
    ap.add_argument("--precision", choices=("fp64", "mixed"), default="fp64")
    ap.add_argument("--steps", type=int, default=None, help="steps to run (default: maxLoop - loop)")
    ap.add_argument("--out", default=None, help="write Vm, activation times and printed rows to this .npz")
    ap.add_argument("--dir", default=".", help="where checkpoints go (checkpointRate)")
    args = ap.parse_args(argv)
    sim = load(args.files, args.simulate)
    out = sim.run(args.precision, args.steps, out_dir=args.dir)
    for row in out["print"]:
        print("%12d %12.6f %12d %21.13e" % (int(row[0]), row[1], int(row[2]), row[3]))
    if args.out:
        np.savez(args.out, **{k: np.asarray(v) for k, v in out.items() if k != "checkpoints"})
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
