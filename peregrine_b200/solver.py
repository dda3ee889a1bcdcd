"""The case driver: the reference's solver API over the native library.

``get_backend``, ``get_solver`` and ``Solver`` keep the reference's names and
calls (peregrine/run.py:6-8, peregrine/backend/__init__.py:8,
peregrine/multiblock/solver.py:23-391): ``step(dt)``, ``rhs(Q=, dQ=)``,
``set_prims``, ``regs``, ``blocks[i].<array>.get() / set()``, ``tme``,
``nrt``, ``run()``.  The arrays, their halos, the kernels and the CUDA graphs
live in the library (include/pgb200.h); this module fills a case from the
config, the mixture and the mesh and forwards the calls.
"""

import ctypes

import numpy as np

from peregrine_b200 import bcs as bcmod
from peregrine_b200 import native
from peregrine_b200.config import ConfigError
from peregrine_b200.grid import metrics as make_metrics
from peregrine_b200.integrators import Integrator, stage_records
from peregrine_b200.iovars import Simulator
from peregrine_b200.mixture import Mixture

NG = 2


class Backend:
    """One device, as the reference's device backend (peregrine/backend/device/backend.py:50-80)."""

    name = "b200"

    def __init__(self, config=None, device=0):
        self.config = config
        self.device = device
        native.load()
        count = ctypes.c_int(0)
        native.call("pgb_device_count", ctypes.byref(count))
        if count.value == 0:
            raise native.PgbCudaError("no CUDA device: this backend runs on a B200 and has no host fallback")
        native.call("pgb_device_init", device)

    def sync(self):
        native.call("pgb_device_sync")

    def stop(self):
        self.sync()


def get_backend(name, config=None, device=0):
    if name not in ("cuda", "b200"):
        raise ValueError(f"{name!r}: this build runs on the device alone (cuda / b200)")
    return Backend(config, device)


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Array:
    """A register of one block, on the device; get/set the reference's host shape."""

    def __init__(self, solver, blk, reg):
        self.solver, self.blk, self.reg = solver, blk, reg

    @property
    def shape(self):
        b = self.solver.blocks[self.blk]
        return tuple(n + 2 * NG for n in b.cells) + (self.solver.ne,)

    def get(self):
        """The full-shaped host array, halo included: what the last right-hand
        side left there (exchanged, or set by a boundary); the halo's edges and
        corners are never read."""
        full = np.empty(self.shape, order="F")
        native.call("pgb_array_get_full", self.solver.case, self.blk, self.reg, _fptr(full), full.size)
        return np.ascontiguousarray(full)

    def set(self, values):
        b = self.solver.blocks[self.blk]
        values = np.asarray(values, dtype=np.float64)
        inner = values[b.interior] if values.shape == self.shape else values
        inner = np.asfortranarray(inner)
        native.call("pgb_array_set", self.solver.case, self.blk, self.reg, _fptr(inner), inner.size)


class SolverBlock:
    def __init__(self, solver, blk):
        self.solver, self.blk = solver, blk
        self.mesh = blk
        for name, reg in solver.regnum.items():
            setattr(self, name, Array(solver, blk.nblki, reg))

    def __getattr__(self, name):
        return getattr(self.mesh, name)


class Solver:
    def __init__(self, cfg, mesh, backend, state=None):
        cfg.validate()
        self.cfg, self.mesh, self.backend = cfg, mesh, backend
        sim = cfg["simulation"]
        self.nrt, self.tme = 0, 0.0
        self.mixture = Mixture(cfg["mixture"])
        self.ns = self.mixture.ns
        # every bcvals entry, checked whether or not a face names it
        self.bcs = bcmod.entries(cfg["bcvals"], sim["simulator"], self.mixture.spnames)
        self.ne = 4 + self.ns
        self.sim = Simulator(self)
        self.integrator = cfg["time-integration"]["integrator"]
        self.integ = Integrator(cfg)
        records, nregs = stage_records(self.integrator)
        self.nregs = nregs
        self.regs = tuple(["Q"] + [f"Q{n}" for n in range(1, nregs)])
        self.regnum = {name: n for n, name in enumerate(self.regs)}
        launch = cfg["backend-b200"]["launch"]
        self.path = {"batched": native.PATH_BATCHED, "per-block": native.PATH_PER_BLOCK,
                     "packed": native.PATH_PACKED}[launch]
        self.graph = bool(cfg["backend-b200"]["graph"])
        adv = cfg["adv-flux"]
        phys = native.Physics()
        phys.simulator = {"euler": native.EULER, "navier-stokes": native.NAVIER_STOKES,
                          "euler-df": native.EULER_DF,
                          "navier-stokes-df": native.NAVIER_STOKES_DF}[sim["simulator"]]
        phys.eos = {"cpg": native.EOS_CPG, "tpg": native.EOS_TPG, "real-gas": native.EOS_REALGAS,
                    "real-gas-df": native.EOS_REALGAS_DF}[cfg["mixture"]["eos"]]
        phys.primary = {"kepaec": native.FLUX_KEPAEC, "hllc": native.FLUX_HLLC, "rusanov": native.FLUX_RUSANOV,
                        "ausmup": native.FLUX_AUSMUP}[adv["primary"]]
        phys.recon = native.RECON_CONSTANT if adv["recon"] == "constant" else native.RECON_MUSCL
        phys.limiter = native.LIMITERS[adv["limiter"]] if adv["recon"] == "muscl" else 0
        trans = cfg["mixture"]["trans"]
        phys.trans = {None: native.TRANS_NONE, "constant": native.TRANS_CONSTANT,
                      "kinetic-theory": native.TRANS_KINETIC}[trans]
        phys.ns = self.ns
        phys.nregs = nregs
        phys.alpha = float(cfg["diff-flux"]["values"].get("alpha", 1.0))
        kind = cfg["chem-integration"]["kind"]
        phys.chemistry = {None: native.CHEM_NONE, "coupled": native.CHEM_COUPLED,
                          "sub-stepped": native.CHEM_SUBSTEPPED}[kind]
        handle = ctypes.c_void_p()
        native.call("pgb_case_create", ctypes.byref(phys), ctypes.byref(handle))
        self.case = handle
        try:
            self._fill(records)
        except Exception:
            native.call("pgb_case_destroy", self.case)
            self.case = None
            raise
        if self.path == native.PATH_BATCHED and self.batched_form() == 0:
            # the batched path takes the ideal gases without boundaries (the
            # fused stage kernel or the fused passes); other physics runs the
            # per-block kernels, still on the device, packed (each pass one
            # launch over every block, the same bits)
            self.path = native.PATH_PACKED
        if state is None:
            self._uniform_ics()

    @property
    def has_bcs(self):
        # a face joined to another rank's block (a shard's, peregrine_b200/shard.py) is traded, not a boundary
        return any(face.nbr is None and getattr(face, "remote", None) is None
                   for blk in self.mesh_blocks for face in blk.intfaces)

    def generated_chemistry(self):
        """Whether the coupled source runs the kernel generated for the
        mechanism, and why not when it does not."""
        on, why = ctypes.c_int(), ctypes.create_string_buffer(512)
        native.call("pgb_case_generated_chemistry", self.case, ctypes.byref(on), why, 512)
        return bool(on.value), why.value.decode()

    def batched_form(self):
        """The batched path's form for this case: 1 the fused stage kernel
        (the single-species calorically perfect kepaec case), 2 the fused
        passes (the other ideal-gas cases without boundaries), 0 neither."""
        form = ctypes.c_int()
        native.call("pgb_case_batched_form", self.case, ctypes.byref(form))
        return form.value

    def fused_capable(self):
        return self.batched_form() > 0

    def species_tables(self):
        """The named species tables the case takes (pgb_case_set_table), from
        the mixture's constants."""
        consts = self.mixture.constants()
        tables = dict(Rsp=consts["Rsp"], h298R=consts["h298R"], MWinv=consts["MWinv"],
                      hpoly0=np.asarray(consts["hpoly"])[:, 0], h298=consts["h298"])
        for key in ("cp0", "mu0", "kappa0", "MWqinv", "wilkepair", "lewis"):
            if key in consts:
                tables[key] = consts[key]
        if self.mixture.eos != "cpg":
            tables.update(cppolyR=consts["cppolyR"], hpoly=consts["hpoly"])
        if self.mixture.eos in ("real-gas", "real-gas-df"):
            for key in ("cubicu", "cubicw", "cubicsigma", "cubiceps", "cubicsqrtac", "cubicb", "cubicda", "cubicmTc",
                        "cubiconepm", "vshift", "cubicsqrtacMW", "cubicbMW", "cubicdaMW", "vshiftMW"):
                tables[key] = np.atleast_1d(consts[key])
        if self.mixture.trans == "kinetic-theory":
            tables.update(mupoly=consts["mupoly"], kappapoly=consts["kappapoly"])
        if self.cfg["chem-integration"]["kind"] == "sub-stepped":
            tables.update(cppoly=consts["cppoly"], MW=consts["MW"])
        if self.mixture.trans is not None and self.cfg["mixture"]["mixing-rule"] == "herning":
            tables["sqrtMW"] = np.sqrt(1.0 / np.asarray(consts["MWinv"], dtype=np.float64))
        if self.mixture.trans is not None and getattr(self.mixture, "diffusion", "lewis") == "binary":
            tables.update(pairfit=consts["pairfit"], selffit=consts["selffit"], bath=consts["bath"], MW=consts["MW"])
        return tables

    def _fill(self, records):
        consts = self.mixture.constants()
        tables = self.species_tables()
        for name, values in tables.items():
            v = np.ascontiguousarray(values, dtype=np.float64).ravel()
            native.call("pgb_case_set_table", self.case, name.encode(), _fptr(v), v.size)
        self.mesh_blocks = self.mesh.make_blocks(NG)
        for blk in self.mesh_blocks:
            out = ctypes.c_int()
            native.call("pgb_case_add_block", self.case, *blk.cells, ctypes.byref(out))
        for blk in self.mesh_blocks:
            for face in blk.intfaces:
                nbr = -1 if face.nbr is None else face.nbr
                rot = getattr(face, "rot", None)
                if face.nbr is not None and (face.orient != "123" or rot is not None):
                    r = None if rot is None else _fptr(np.ascontiguousarray(rot, dtype=np.float64).ravel())
                    native.call("pgb_case_connect_oriented", self.case, blk.nblki, face.nface, nbr,
                                face.orient.encode(), r)
                else:
                    native.call("pgb_case_connect", self.case, blk.nblki, face.nface, nbr, face.nbrface or 0)
        self._fill_bcs()
        chem = self.cfg["chem-integration"]
        if chem["kind"] is not None:
            mech, keep = native.mechanism(consts)
            native.call("pgb_case_set_mechanism", self.case, ctypes.byref(mech))
        if chem["kind"] == "sub-stepped":
            native.call("pgb_case_set_substeps", self.case, chem["max-substeps"], chem["bulk-substeps"],
                        chem["stiff-bins"], float(chem["equilibrium-tolerance"]))
        native.call("pgb_case_set_stages", self.case, records, len(records))
        # the coupled source generated for the mechanism, or the table-driven kernel
        generated = self.cfg["backend-b200"]["chemistry-kernel"] == "generated"
        native.call("pgb_case_set_generated_chemistry", self.case, 1 if generated else 0)
        native.call("pgb_case_finalize", self.case)
        self.metrics = []
        for blk in self.mesh_blocks:
            m = make_metrics(blk.nodes, NG)
            self.metrics.append(m)
            for name, arr in m.items():
                a = np.asarray(arr, dtype=np.float64)
                a = np.asfortranarray(a.reshape(a.shape[:3] + (-1,)))
                native.call("pgb_metric_set", self.case, blk.nblki, native.METRIC_IDS[name], _fptr(a), a.size)
        self.blocks = [SolverBlock(self, b) for b in self.mesh_blocks]

    def _fill_bcs(self):
        """The bcvals entries and the boundary faces that name them."""
        bcmod.check_faces(self.mesh_blocks, self.cfg["bcvals"])
        ids = {}
        for name, entry in self.bcs.items():
            kind, ops, args, starts = entry.program()
            o = (ctypes.c_int * max(1, len(ops)))(*ops)
            a = (ctypes.c_double * max(1, len(args)))(*args)
            st = (ctypes.c_int * len(starts))(*starts)
            out = ctypes.c_int()
            native.call("pgb_case_add_bc", self.case, kind, o, a, st, len(entry.values), ctypes.byref(out))
            ids[name] = out.value
        for blk in self.mesh_blocks:
            for face in blk.intfaces:
                if face.nbr is None and getattr(face, "remote", None) is None:
                    native.call("pgb_case_set_face_bc", self.case, blk.nblki, face.nface, ids[face.bcname])

    def __del__(self):
        case = getattr(self, "case", None)
        if case:
            try:
                native.call("pgb_case_destroy", case)
            except Exception:
                pass
            self.case = None

    # the reference's ics section: a uniform state of p, u, v, w, T, Y
    def _uniform_ics(self):
        ic = self.cfg["ics"]
        names = self.mixture.spnames
        unknown = sorted(set(ic["Y"]) - set(names))
        if unknown:
            raise ConfigError("ics.Y", f"names {unknown}, which are not species of this mixture: {names}.")
        values = [ic[k] for k in ("p", "u", "v", "w", "T")] + [ic["Y"].get(n, 0.0) for n in names[:-1]]
        prims = []
        for b in self.mesh_blocks:
            q = np.empty(tuple(n + 2 * NG for n in b.cells) + (self.ne,))
            q[...] = values
            prims.append(q)
        self.set_prims(prims)

    ###########################################################################
    # The reference's per-step API
    ###########################################################################
    def set_prims(self, prims):
        """Q from primitive arrays, one per block: p, u, v, w, T, Y... in the last axis."""
        for b, q in zip(self.mesh_blocks, prims):
            q = np.asarray(q, dtype=np.float64)
            full = tuple(n + 2 * NG for n in b.cells) + (self.ne,)
            inner = q[b.interior] if q.shape == full else q
            if inner.shape != b.cells + (self.ne,):
                raise ValueError(f"block {b.nblki}: primitives of shape {q.shape}")
            inner = np.asfortranarray(inner)
            native.call("pgb_set_prims", self.case, b.nblki, 0, _fptr(inner), inner.size)

    def advance(self, n):
        """Stage n's combines on the registers as they are, after its
        right-hand side (peregrine/multiblock/solver.py:276-280); the step
        size is ``dt``'s."""
        native.call("pgb_advance", self.case, int(n))

    def prerhs(self, Q="Q", dQ=None):
        """Register Q readied for reading: its halo, state and boundary halo
        cells formed (peregrine/multiblock/solver.py:246-250).  The library
        forms them in a right-hand side of the per-block kernels, which keep
        the state array, into dQ (the last register unless named), as the
        reference's prerhs begins dQ."""
        if self.has_bcs:
            native.call("pgb_set_time", self.case, float(self.tme))
        native.call("pgb_rhs", self.case, self.regnum[Q], self.regnum[dQ or self.regs[-1]])

    def postrhs(self, Q=None):
        """Register Q (the solution unless named) readied after it was written
        (peregrine/multiblock/solver.py:282-285)."""
        self.prerhs(Q or "Q")

    @property
    def dt(self):
        """The step scalar, read and set as the reference's ``mb.dt``."""
        return _DeviceScalar(self.last_dt, self.set_dt)

    def exchange(self, Q="Q"):
        """Register Q's halo filled across every interface, a rotationally
        periodic face's vectors turned (the reference's exchange of a bank)."""
        native.call("pgb_exchange", self.case, self.regnum[Q])

    def rhs(self, *, Q="Q", dQ=None):
        """dQ of register Q on the case's path: on the batched path the fused
        stage kernel itself, writing the dQ it forms (at unit step and no
        register term), on the others the per-block kernels."""
        dQ = dQ or self.regs[-1]
        if self.has_bcs:
            native.call("pgb_set_time", self.case, float(self.tme))
        native.call("pgb_rhs_path", self.case, self.regnum[Q], self.regnum[dQ], self.path)

    def step(self, dt, nsteps=1):
        # the boundaries read the clock from the step's start on
        if self.has_bcs:
            native.call("pgb_set_time", self.case, float(self.tme))
        native.call("pgb_step", self.case, float(dt), int(nsteps), self.path, int(self.graph))
        self.nrt += nsteps
        self.tme += dt * nsteps

    def run(self):
        """niter steps under the config's controller (peregrine/multiblock/solver.py:366-370).
        Under the cfl controller each step's size is worked out on the device
        from the step's own start, so the steps queue without a host round
        trip; the clock is read back at the end."""
        sim = self.cfg["simulation"]
        n = sim["niter"]
        if sim["controller"] == "cfl":
            self.step_cfl(sim["cfl"], sim["dt-max"], n)
        else:
            self.step(sim["dt"], n)
        self.backend.sync()

    def step_cfl(self, cfl, dtmax, nsteps=1):
        native.call("pgb_set_time", self.case, float(self.tme))
        native.call("pgb_step_cfl", self.case, float(cfl), float(dtmax), int(nsteps), self.path, int(self.graph))
        self.nrt += nsteps
        t = ctypes.c_double()
        native.call("pgb_get_time", self.case, ctypes.byref(t))
        self.tme = t.value

    def cflmax(self):
        """The largest acoustic, convective and combined CFL number per unit
        step over every block's interior of Q (peregrine/multiblock/solver.py:292-296)."""
        out = (ctypes.c_double * 3)()
        native.call("pgb_cflmax", self.case, 0, out)
        return dict(zip(("acoustic", "convective", "combined"), list(out)))

    def substeps(self, blk=0):
        """Each interior cell's substep count at the last right-hand side (the
        reference's ``substeps`` array)."""
        b = self.mesh_blocks[blk]
        out = np.zeros(b.cells, dtype=np.int32, order="F")
        native.call("pgb_substeps_get", self.case, blk, out.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), out.size)
        return out

    def stiff_head(self):
        """The stiff list's header: the cells listed, then each bin's count."""
        n = self.cfg["chem-integration"]["stiff-bins"] + 1
        out = (ctypes.c_uint * n)()
        native.call("pgb_stiff_head", self.case, out, n)
        return list(out)

    def set_dt(self, dt):
        """The step scalar the sub-stepped chemistry integrates over (the
        reference's ``solver.dt``), for a right-hand side outside a step."""
        native.call("pgb_set_dt", self.case, float(dt))

    def last_dt(self):
        dt = ctypes.c_double()
        native.call("pgb_last_dt", self.case, ctypes.byref(dt))
        return dt.value

    def last_step_ms(self):
        ms = ctypes.c_float()
        native.call("pgb_last_step_ms", self.case, ctypes.byref(ms))
        return ms.value

    def launches_per_step(self, path=None):
        n = ctypes.c_int()
        native.call("pgb_launches_per_step", self.case, self.path if path is None else path, ctypes.byref(n))
        return n.value

    def set_tile(self, blk, tw, th, kchunk):
        native.call("pgb_set_tile", self.case, blk, tw, th, kchunk)

    def get_tile(self, blk):
        v = [ctypes.c_int() for _ in range(3)]
        native.call("pgb_get_tile", self.case, blk, *[ctypes.byref(x) for x in v])
        return tuple(x.value for x in v)

    def uniform(self, blk):
        u = ctypes.c_int()
        native.call("pgb_block_uniform", self.case, blk, ctypes.byref(u))
        return bool(u.value)

    def stream(self):
        s = ctypes.c_void_p()
        native.call("pgb_case_stream", self.case, ctypes.byref(s))
        return s.value

    @property
    def ncells(self):
        return sum(b.ncells for b in self.mesh_blocks)


class _DeviceScalar:
    """A device scalar's get and set (the reference's Scalar)."""

    def __init__(self, get, set_):
        self.get, self.set = get, set_


def get_solver(cfg, mesh, backend, state=None, cls=Solver):
    return cls(cfg, mesh, backend, state)
