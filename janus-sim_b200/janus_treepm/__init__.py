"""Host-side mirror of the janus-sim TreePM interface over the B200 engine.

The engine is libjanus_treepm.so (CUDA for sm_100a, built in-tree by
`make -C janus-sim_b200`); this module binds its C ABI (include/janus_treepm.h)
with ctypes and offers the reference's two call shapes:

* ``GpuNBodyTwoPass`` -- src/nbody_gpu_twopass.rs: ``with_custom_ics(pos, vel,
  signs, box_size)``, ``set_theta``, ``set_softening``, ``set_mass_factor``,
  ``set_pm_k_min``, ``step_treepm_gpu(dt, r_cut, hubble, dtau_per_dt)``,
  ``compute_forces()``, ``get_particles()``.
* ``TreePMForce`` -- src/treepm/treepm_force.rs: ``TreePMForce(r_cut,
  grid_size, box_size, theta, softening)``, ``update(particles)``,
  ``compute_all_forces(particles)``.

Errors raise ``JanusError`` carrying the library's negative code (the
reference returns ``Result<_, Box<dyn Error>>``).  There is no CPU fallback:
if the library is missing or no CUDA device is present, every call raises.
"""
import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
# JANUS_TREEPM_LIB selects another build of the same library (for A/B timing)
LIB_PATH = os.environ.get("JANUS_TREEPM_LIB", os.path.join(PKG_ROOT, "libjanus_treepm.so"))

JT_OK, JT_EINVAL, JT_ENOMEM, JT_ECUDA, JT_ETIMEDOUT = 0, -1, -2, -3, -4
JT_ENOTIMPL, JT_ESTATE, JT_EOVERFLOW, JT_EBUSY = -5, -6, -7, -8
JT_MEM_HOST, JT_MEM_DEVICE = 0, 1
JT_ACCURATE, JT_RCOMPAT = 0, 1
JT_KDK, JT_DKD_REF = 0, 1
JT_PART_PM, JT_PART_SHORT, JT_PART_ALL = 1, 2, 3

EXPORTED = [
    "jt_create", "jt_set_state", "jt_set_state_signed", "jt_accel", "jt_accel_signed",
    "jt_step", "jt_get_state", "jt_get_state_signed", "jt_debug_tree", "jt_get_timings",
    "jt_counts", "jt_destroy", "jt_strerror", "jt_version", "jt_fp32_peak", "jt_accel_part",
    "jt_walk_counters",
    "jt_batch_create", "jt_batch_destroy", "jt_batch_add", "jt_batch_remove", "jt_batch_forces",
    "jt_batch_step", "jt_batch_get_accel", "jt_batch_get_state", "jt_batch_box_info",
    "jt_batch_memory", "jt_batch_estimate", "jt_batch_get_timings", "jt_morton_sort_static",
    "jt_batch_trim", "jt_batch_set_graphs", "jt_server_create", "jt_server_destroy",
    "jt_server_add_job", "jt_server_request", "jt_server_clock", "jt_server_poll", "jt_server_serve",
    "jt_server_job_state", "jt_server_get_state", "jt_server_stats", "jt_server_job_need",
    "jt_walk_tuning", "jt_wait_probe", "jt_diagnostics", "jt_batch_diagnostics",
    "jt_snapshot_write", "jt_snapshot_read", "jt_checkpoint", "jt_set_screening",
    "jt_ics_zeldovich", "jt_set_state_zeldovich", "jt_batch_add_zeldovich", "jt_philox4x32_10",
    "jt_energy_sampled", "jt_virialize_sampled", "jt_energy_drift_pct",
    "jt_batch_checkpoint_async", "jt_batch_checkpoint_wait", "jt_snapshot_write_raw",
    "jt_snapshot_read_raw", "jt_set_accel", "jt_get_accel", "jt_server_get_accel",
    "jt_batch_set_screening", "jt_step_host", "jt_batch_prepare", "jt_config_short_cut",
    "jt_expansion_create", "jt_expansion_destroy", "jt_expansion_info", "jt_expansion_at_time",
    "jt_expansion_at_redshift", "jt_expansion_state_at_mu", "jt_expansion_calibrate",
    "jt_expansion_phi_factors", "jt_server_get_timings", "jt_set_counters", "jt_batch_set_counters",
    "jt_server_set_counters",
]
JT_JOB_QUEUED, JT_JOB_RESIDENT, JT_JOB_DONE = 0, 1, 2
JT_STATIC_SORT_MAX = 262144


class JanusError(RuntimeError):
    def __init__(self, code, what=""):
        self.code = code
        msg = _strerror(code)
        super().__init__(f"{what}: {msg} ({code})" if what else f"{msg} ({code})")


class jt_config(C.Structure):
    _fields_ = [
        ("box_L", C.c_double), ("pm_grid", C.c_int), ("theta", C.c_double),
        ("softening", C.c_double), ("r_s", C.c_double), ("r_cut", C.c_double),
        ("mu", C.c_double), ("G_mass_plus", C.c_double), ("k_min", C.c_int),
        ("mode", C.c_int), ("integrator", C.c_int), ("pm_order", C.c_int),
        ("pm_interlace", C.c_int), ("cut_tail_ppm", C.c_int), ("reserved", C.c_int * 2),
    ]


class jt_timings(C.Structure):
    _fields_ = [
        ("sort_ms", C.c_double), ("tree_ms", C.c_double), ("deposit_ms", C.c_double),
        ("fft_ms", C.c_double), ("kspace_ms", C.c_double), ("walk_ms", C.c_double),
        ("kick_drift_ms", C.c_double), ("total_ms", C.c_double),
        ("interactions", C.c_int64), ("launches", C.c_int64),
        ("pair_interactions", C.c_int64), ("node_interactions", C.c_int64),
        ("candidates", C.c_int64), ("cellwalk_ms", C.c_double), ("interp_ms", C.c_double),
    ]


class jt_expansion_state(C.Structure):
    _fields_ = [("mu", C.c_double), ("a_plus", C.c_double), ("t_gyr", C.c_double),
                ("h_plus", C.c_double), ("z", C.c_double)]

    def to_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class jt_expansion_info_t(C.Structure):
    _fields_ = [("alpha", C.c_double), ("mu_0", C.c_double), ("a_0", C.c_double), ("z_max", C.c_double),
                ("z_init", C.c_double), ("t_start", C.c_double), ("t_end", C.c_double),
                ("n_points", C.c_int64)]


class jt_step_args(C.Structure):
    _fields_ = [("dt", C.c_double), ("hubble", C.c_double), ("dtau_per_dt", C.c_double)]


class jt_diag(C.Structure):
    _fields_ = [
        ("segregation", C.c_double), ("diff_over_poisson", C.c_double), ("corr", C.c_double),
        ("exc_var_minus", C.c_double), ("kinetic", C.c_double * 2), ("momentum", C.c_double * 6),
        ("com", C.c_double * 6),
    ]

    def to_dict(self):
        return {"segregation": self.segregation, "diff_over_poisson": self.diff_over_poisson,
                "corr": self.corr, "exc_var_minus": self.exc_var_minus,
                "kinetic": list(self.kinetic),
                "momentum": [list(self.momentum[0:3]), list(self.momentum[3:6])],
                "com": [list(self.com[0:3]), list(self.com[3:6])]}


class jt_snapshot_meta(C.Structure):
    _fields_ = [("a", C.c_double), ("t_gyr", C.c_double), ("h0", C.c_double), ("omega_b", C.c_double),
                ("z_init", C.c_double), ("z_start_run", C.c_double), ("seed_ic", C.c_uint32),
                ("run_label", C.c_char * 256)]


def snapshot_meta(a=1.0, t_gyr=0.0, h0=69.9, omega_b=0.05, z_init=10.0, z_start_run=10.0, seed_ic=42,
                  run_label=""):
    m = jt_snapshot_meta()
    m.a, m.t_gyr, m.h0, m.omega_b, m.z_init, m.z_start_run = a, t_gyr, h0, omega_b, z_init, z_start_run
    m.seed_ic = seed_ic
    m.run_label = run_label.encode()[:255]
    return m


def snapshot_write(path, meta, box_L, mu, pos, vel, signs, mass, eps):
    """Write the reference's snapshot_v3 file (host arrays)."""
    pos = _f32(pos)
    vel = None if vel is None else _f32(vel)
    signs = np.ascontiguousarray(signs, np.int8)
    mass = np.ascontiguousarray(mass, np.float32)
    eps = np.ascontiguousarray(eps, np.float32)
    _check(library().jt_snapshot_write(str(path).encode(), C.byref(meta), box_L, mu, _ptr(pos), _ptr(vel),
                                       _ptr(signs), _ptr(mass), _ptr(eps), len(pos)), "jt_snapshot_write")


def snapshot_read(path):
    """Read a snapshot_v3 file: (meta, box_L, mu, pos, vel, signs, mass, eps)."""
    L = library()
    meta, box, mu, n = jt_snapshot_meta(), C.c_double(), C.c_double(), C.c_size_t()
    _check(L.jt_snapshot_read(str(path).encode(), C.byref(meta), C.byref(box), C.byref(mu), None, None,
                              None, None, None, 0, C.byref(n)), "jt_snapshot_read")
    k = n.value
    pos, vel = np.zeros((k, 3), np.float32), np.zeros((k, 3), np.float32)
    sg, mass, eps = np.zeros(k, np.int8), np.zeros(k, np.float32), np.zeros(k, np.float32)
    _check(L.jt_snapshot_read(str(path).encode(), C.byref(meta), C.byref(box), C.byref(mu), _ptr(pos),
                              _ptr(vel), _ptr(sg), _ptr(mass), _ptr(eps), k, C.byref(n)), "jt_snapshot_read")
    return meta, box.value, mu.value, pos, vel, sg, mass, eps


class jt_energy(C.Structure):
    _fields_ = [("kinetic", C.c_double), ("pe_binding", C.c_double), ("pe_plus", C.c_double),
                ("pe_minus", C.c_double), ("n_sampled", C.c_int64 * 2)]

    def to_dict(self):
        return dict(kinetic=self.kinetic, pe_binding=self.pe_binding, pe_plus=self.pe_plus,
                    pe_minus=self.pe_minus, n_sampled=tuple(self.n_sampled))


def energy_drift_pct(e_now, e_initial):
    return library().jt_energy_drift_pct(e_now, e_initial)


class jt_ics_params(C.Structure):
    _fields_ = [("n_side", C.c_int), ("box_L", C.c_double), ("seed", C.c_uint64),
                ("rms_frac", C.c_double), ("vel_factor", C.c_double)]


def ics_params(n_side, box_L, seed=42, rms_frac=0.3, vel_factor=0.05):
    p = jt_ics_params()
    p.n_side, p.box_L, p.seed, p.rms_frac, p.vel_factor = n_side, box_L, seed, rms_frac, vel_factor
    return p


def zeldovich_device(n_side, box_L, seed=42, rms_frac=0.3, vel_factor=0.05):
    """Zel'dovich lattice ICs generated on the current device; returns host
    (pos_p, vel_p, pos_m, vel_m), n_side^3 rows each."""
    n3 = n_side ** 3
    out = [np.zeros((n3, 3), np.float32) for _ in range(4)]
    p = ics_params(n_side, box_L, seed, rms_frac, vel_factor)
    _check(library().jt_ics_zeldovich(C.byref(p), *[_ptr(a) for a in out], JT_MEM_HOST),
           "jt_ics_zeldovich")
    return tuple(out)


def philox4x32_10(ctr, key):
    """The IC generator's counter-based stream (host copy)."""
    c = (C.c_uint * 4)(*ctr)
    k = (C.c_uint * 2)(*key)
    o = (C.c_uint * 4)()
    library().jt_philox4x32_10(c, k, o)
    return tuple(o)


def snapshot_write_raw(path, pos, vel, signs, box_L, step, z):
    """The production driver's raw snapshot (25-byte records)."""
    pos = _f32(pos)
    vel = None if vel is None else _f32(vel)
    signs = np.ascontiguousarray(signs, np.int8)
    _check(library().jt_snapshot_write_raw(str(path).encode(), _ptr(pos), _ptr(vel), _ptr(signs),
                                           len(pos), box_L, step, z), "jt_snapshot_write_raw")


def snapshot_read_raw(path):
    """(pos, vel, signs, box_L, step, z) of a raw snapshot."""
    L = library()
    n, box, st, z = C.c_size_t(), C.c_double(), C.c_uint32(), C.c_double()
    _check(L.jt_snapshot_read_raw(str(path).encode(), None, None, None, 0, C.byref(n), C.byref(box),
                                  C.byref(st), C.byref(z)), "jt_snapshot_read_raw")
    k = n.value
    pos, vel, sg = np.zeros((k, 3), np.float32), np.zeros((k, 3), np.float32), np.zeros(k, np.int8)
    _check(L.jt_snapshot_read_raw(str(path).encode(), _ptr(pos), _ptr(vel), _ptr(sg), k, C.byref(n),
                                  C.byref(box), C.byref(st), C.byref(z)), "jt_snapshot_read_raw")
    return pos, vel, sg, box.value, st.value, z.value


class jt_serve_stats(C.Structure):
    _fields_ = [
        ("requests_served", C.c_int64), ("batched_steps", C.c_int64), ("particle_steps", C.c_int64),
        ("admitted", C.c_int64), ("evicted", C.c_int64), ("admission_waits", C.c_int64),
        ("p50_latency_s", C.c_double), ("p99_latency_s", C.c_double), ("max_latency_s", C.c_double),
        ("busy_s", C.c_double), ("peak_device_bytes", C.c_int64), ("max_jobs_per_step", C.c_int64),
        ("swapped_out", C.c_int64), ("trims", C.c_int64), ("admit_s", C.c_double),
        ("evict_s", C.c_double), ("step_device_s", C.c_double), ("reserved_gb", C.c_double),
    ]


_lib = None


def library():
    """Load libjanus_treepm.so (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} not built: run `make -C janus-sim_b200`")
    L = C.CDLL(LIB_PATH)
    vp, fp, i8p = C.c_void_p, C.c_void_p, C.c_void_p
    H = C.c_void_p
    L.jt_create.argtypes = [C.POINTER(jt_config), C.POINTER(H)]
    L.jt_set_state.argtypes = [H, fp, fp, C.c_size_t, fp, fp, C.c_size_t, C.c_int]
    L.jt_set_state_signed.argtypes = [H, fp, fp, i8p, C.c_size_t, C.c_int]
    L.jt_accel.argtypes = [H, fp, fp, C.c_int]
    L.jt_accel_signed.argtypes = [H, fp, C.c_int]
    L.jt_accel_part.argtypes = [H, C.c_int, fp, fp, C.c_int]
    L.jt_step.argtypes = [H, C.c_double, C.c_double, C.c_double, C.c_int]
    L.jt_get_state.argtypes = [H, fp, fp, fp, fp, C.c_int]
    L.jt_get_state_signed.argtypes = [H, fp, fp, C.c_int]
    L.jt_debug_tree.argtypes = [H, C.c_int, vp, vp, vp, vp, vp]
    L.jt_get_timings.argtypes = [H, C.POINTER(jt_timings)]
    L.jt_counts.argtypes = [H, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]
    L.jt_destroy.argtypes = [H]
    L.jt_destroy.restype = None
    L.jt_strerror.argtypes = [C.c_int]
    L.jt_strerror.restype = C.c_char_p
    L.jt_fp32_peak.argtypes = [C.c_int, C.POINTER(C.c_double)]
    L.jt_config_short_cut.argtypes = [C.POINTER(jt_config), C.POINTER(C.c_double)]
    dp_ = C.POINTER(C.c_double)
    L.jt_expansion_create.argtypes = [C.c_double, C.c_int, C.POINTER(H)]
    L.jt_expansion_destroy.argtypes = [H]
    L.jt_expansion_destroy.restype = None
    L.jt_expansion_info.argtypes = [H, C.POINTER(jt_expansion_info_t)]
    L.jt_expansion_at_time.argtypes = [H, C.c_double, C.POINTER(jt_expansion_state)]
    L.jt_expansion_at_redshift.argtypes = [H, C.c_double, C.POINTER(jt_expansion_state)]
    L.jt_expansion_state_at_mu.argtypes = [C.c_double, C.c_double, C.c_double,
                                           C.POINTER(jt_expansion_state)]
    L.jt_expansion_calibrate.argtypes = [dp_, dp_]
    L.jt_expansion_phi_factors.argtypes = [C.c_double, C.c_double, dp_, dp_, dp_]
    L.jt_walk_counters.argtypes = [H, C.POINTER(C.c_int64)]
    L.jt_version.argtypes = []
    L.jt_version.restype = C.c_char_p
    szp = C.POINTER(C.c_size_t)
    L.jt_batch_create.argtypes = [C.POINTER(H)]
    L.jt_batch_destroy.argtypes = [H]
    L.jt_batch_destroy.restype = None
    L.jt_batch_add.argtypes = [H, C.POINTER(jt_config), fp, fp, C.c_size_t, fp, fp, C.c_size_t, C.c_int,
                               C.POINTER(C.c_int)]
    L.jt_batch_remove.argtypes = [H, C.c_int]
    L.jt_batch_forces.argtypes = [H, C.POINTER(C.c_int), C.c_int, C.c_int]
    L.jt_batch_step.argtypes = [H, C.POINTER(C.c_int), C.c_int, C.POINTER(jt_step_args), C.c_int]
    L.jt_batch_get_accel.argtypes = [H, C.c_int, fp, fp, C.c_int]
    L.jt_batch_get_state.argtypes = [H, C.c_int, fp, fp, fp, fp, C.c_int]
    L.jt_batch_box_info.argtypes = [H, C.c_int, szp, szp, szp]
    L.jt_batch_memory.argtypes = [H, szp, szp]
    L.jt_batch_estimate.argtypes = [C.POINTER(jt_config), C.c_size_t, C.c_size_t, szp, szp]
    L.jt_batch_get_timings.argtypes = [H, C.POINTER(jt_timings)]
    L.jt_morton_sort_static.argtypes = [vp, C.c_size_t, C.c_double, vp, vp, vp]
    L.jt_walk_tuning.argtypes = [C.c_char_p, C.c_size_t]
    L.jt_wait_probe.argtypes = [C.c_int, C.POINTER(C.c_int)]
    L.jt_diagnostics.argtypes = [H, C.c_int, C.POINTER(jt_diag)]
    L.jt_snapshot_write.argtypes = [C.c_char_p, C.POINTER(jt_snapshot_meta), C.c_double, C.c_double,
                                    fp, fp, vp, fp, fp, C.c_size_t]
    L.jt_snapshot_read.argtypes = [C.c_char_p, C.POINTER(jt_snapshot_meta), C.POINTER(C.c_double),
                                   C.POINTER(C.c_double), fp, fp, vp, fp, fp, C.c_size_t,
                                   C.POINTER(C.c_size_t)]
    L.jt_checkpoint.argtypes = [H, C.c_char_p, C.POINTER(jt_snapshot_meta)]
    L.jt_set_screening.argtypes = [H, C.c_double, C.c_double]
    L.jt_batch_set_screening.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
    L.jt_step_host.argtypes = [H, fp, fp, fp, fp, fp, fp, C.c_double, C.c_double, C.c_double]
    L.jt_batch_prepare.argtypes = [C.c_void_p, C.c_int]
    L.jt_set_accel.argtypes = [H, fp, fp, C.c_int]
    L.jt_server_get_accel.argtypes = [H, C.c_int, fp, fp]
    L.jt_get_accel.argtypes = [H, fp, fp, C.c_int]
    L.jt_ics_zeldovich.argtypes = [C.POINTER(jt_ics_params), fp, fp, fp, fp, C.c_int]
    L.jt_set_state_zeldovich.argtypes = [H, C.POINTER(jt_ics_params)]
    L.jt_batch_add_zeldovich.argtypes = [C.c_void_p, C.POINTER(jt_config), C.POINTER(jt_ics_params),
                                         C.POINTER(C.c_int)]
    L.jt_philox4x32_10.argtypes = [C.POINTER(C.c_uint), C.POINTER(C.c_uint), C.POINTER(C.c_uint)]
    L.jt_philox4x32_10.restype = None
    L.jt_energy_sampled.argtypes = [H, C.c_size_t, C.POINTER(jt_energy)]
    L.jt_virialize_sampled.argtypes = [H, C.c_size_t, C.POINTER(C.c_double)]
    L.jt_energy_drift_pct.argtypes = [C.c_double, C.c_double]
    L.jt_energy_drift_pct.restype = C.c_double
    L.jt_batch_checkpoint_async.argtypes = [C.c_void_p, C.c_int, C.c_char_p, C.POINTER(jt_snapshot_meta)]
    L.jt_batch_checkpoint_wait.argtypes = [C.c_void_p]
    L.jt_snapshot_write_raw.argtypes = [C.c_char_p, fp, fp, vp, C.c_size_t, C.c_double, C.c_uint32,
                                        C.c_double]
    L.jt_snapshot_read_raw.argtypes = [C.c_char_p, fp, fp, vp, C.c_size_t, C.POINTER(C.c_size_t),
                                       C.POINTER(C.c_double), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_double)]
    L.jt_batch_diagnostics.argtypes = [H, C.c_int, C.c_int, C.POINTER(jt_diag)]
    L.jt_batch_trim.argtypes = [H]
    L.jt_batch_set_graphs.argtypes = [H, C.c_int]
    L.jt_server_create.argtypes = [C.c_size_t, C.POINTER(H)]
    L.jt_server_destroy.argtypes = [H]
    L.jt_server_destroy.restype = None
    L.jt_server_add_job.argtypes = [H, C.POINTER(jt_config), fp, fp, C.c_size_t, fp, fp, C.c_size_t,
                                    C.c_int, C.POINTER(jt_step_args), C.POINTER(C.c_int)]
    L.jt_server_request.argtypes = [H, C.c_int, C.c_double]
    L.jt_server_clock.argtypes = [H]
    L.jt_server_clock.restype = C.c_double
    L.jt_server_poll.argtypes = [H, C.POINTER(C.c_int)]
    L.jt_server_serve.argtypes = [H, vp, vp, C.c_int]
    L.jt_server_job_state.argtypes = [H, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.jt_server_get_state.argtypes = [H, C.c_int, fp, fp, fp, fp]
    L.jt_server_stats.argtypes = [H, C.POINTER(jt_serve_stats)]
    L.jt_server_get_timings.argtypes = [H, C.POINTER(jt_timings)]
    L.jt_set_counters.argtypes = [H, C.c_int]
    L.jt_batch_set_counters.argtypes = [H, C.c_int]
    L.jt_server_set_counters.argtypes = [H, C.c_int]
    L.jt_server_job_need.argtypes = [C.POINTER(jt_config), C.c_size_t, C.c_size_t, C.POINTER(C.c_size_t)]
    for name in EXPORTED:
        if name not in ("jt_destroy", "jt_strerror", "jt_version", "jt_batch_destroy",
                        "jt_server_destroy", "jt_server_clock", "jt_philox4x32_10",
                        "jt_energy_drift_pct", "jt_expansion_destroy"):
            getattr(L, name).restype = C.c_int
    _lib = L
    return L


def _strerror(code):
    try:
        return library().jt_strerror(code).decode()
    except Exception:
        return "error"


def _check(code, what):
    if code != JT_OK:
        raise JanusError(code, what)


def _f32(a, n3=True):
    a = np.ascontiguousarray(a, dtype=np.float32)
    if n3:
        a = a.reshape(-1, 3)
    return a


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


@dataclass
class Config:
    """Solver configuration (the fields of jt_config)."""
    box_L: float
    pm_grid: int
    theta: float = 0.5
    softening: float = 0.1
    r_s: float = 0.0            # 0 -> 1.25 PM cells
    r_cut: float = 0.0          # 0 -> 4.5 r_s
    mu: float = 1.0             # M- / M+
    G_mass_plus: float = 1.0    # G * mass of one m+ particle
    k_min: int = 0
    mode: int = JT_ACCURATE
    integrator: int = JT_KDK
    pm_order: int = 0           # 0 -> PCS (accurate); 2 CIC; 3 TSC; 4 PCS
    pm_interlace: int = 0       # 0 -> on (accurate); 1 on; 2 off
    cut_tail_ppm: int = 0       # > 0: widen the short-range cut until S = ppm * 1e-6

    def resolved(self):
        c = Config(**self.__dict__)
        if c.r_s <= 0:
            c.r_s = 1.25 * c.box_L / c.pm_grid
        if c.r_cut <= 0:
            c.r_cut = 4.5 * c.r_s
        return c

    def to_c(self):
        c = self.resolved()
        s = jt_config()
        s.box_L, s.pm_grid, s.theta, s.softening = c.box_L, c.pm_grid, c.theta, c.softening
        s.r_s, s.r_cut, s.mu, s.G_mass_plus = c.r_s, c.r_cut, c.mu, c.G_mass_plus
        s.k_min, s.mode, s.integrator = c.k_min, c.mode, c.integrator
        s.pm_order, s.pm_interlace = c.pm_order, c.pm_interlace
        s.cut_tail_ppm = c.cut_tail_ppm
        return s


class Solver:
    """One simulation box on the current CUDA device (a jt_handle)."""

    def __init__(self, config: Config):
        self.config = config.resolved()
        self._h = C.c_void_p()
        cfg = self.config.to_c()
        _check(library().jt_create(C.byref(cfg), C.byref(self._h)), "jt_create")
        self._signed = False
        self.n = (0, 0)

    def close(self):
        if self._h:
            library().jt_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- state
    def set_state(self, pos_p, vel_p, pos_m, vel_m):
        pos_p = _f32(pos_p) if pos_p is not None else np.zeros((0, 3), np.float32)
        pos_m = _f32(pos_m) if pos_m is not None else np.zeros((0, 3), np.float32)
        vel_p = None if vel_p is None else _f32(vel_p)
        vel_m = None if vel_m is None else _f32(vel_m)
        _check(library().jt_set_state(self._h, _ptr(pos_p), _ptr(vel_p), len(pos_p), _ptr(pos_m),
                                      _ptr(vel_m), len(pos_m), JT_MEM_HOST), "jt_set_state")
        self._signed = False
        self.n = (len(pos_p), len(pos_m))

    def set_state_signed(self, pos, vel, signs):
        pos = _f32(pos)
        vel = None if vel is None else _f32(vel)
        signs = np.ascontiguousarray(signs, dtype=np.int8)
        _check(library().jt_set_state_signed(self._h, _ptr(pos), _ptr(vel), _ptr(signs), len(pos),
                                             JT_MEM_HOST), "jt_set_state_signed")
        self._signed = True
        n_p = int((signs > 0).sum())
        self.n = (n_p, len(signs) - n_p)

    def set_state_zeldovich(self, n_side, seed=42, rms_frac=0.3, vel_factor=0.05):
        """Zel'dovich lattice ICs generated on the device as the state (box_L
        from the config)."""
        p = ics_params(n_side, self.config.box_L, seed, rms_frac, vel_factor)
        _check(library().jt_set_state_zeldovich(self._h, C.byref(p)), "jt_set_state_zeldovich")
        self._signed = False
        self.n = (n_side ** 3, n_side ** 3)

    def set_state_device(self, pos_p, vel_p, pos_m, vel_m):
        """Device (torch CUDA float32 (n,3) contiguous) tensors; vel may be None."""
        def dp(t):
            return None if t is None else C.c_void_p(t.data_ptr())
        n_p = 0 if pos_p is None else pos_p.shape[0]
        n_m = 0 if pos_m is None else pos_m.shape[0]
        _check(library().jt_set_state(self._h, dp(pos_p), dp(vel_p), n_p, dp(pos_m), dp(vel_m),
                                      n_m, JT_MEM_DEVICE), "jt_set_state")
        self._signed = False
        self.n = (n_p, n_m)

    def accel(self):
        """Accelerations (acc_p (n+,3), acc_m (n-,3)) or, after set_state_signed, one array."""
        if self._signed:
            out = np.zeros((sum(self.n), 3), np.float32)
            _check(library().jt_accel_signed(self._h, _ptr(out), JT_MEM_HOST), "jt_accel_signed")
            return out
        ap = np.zeros((self.n[0], 3), np.float32)
        am = np.zeros((self.n[1], 3), np.float32)
        _check(library().jt_accel(self._h, _ptr(ap), _ptr(am), JT_MEM_HOST), "jt_accel")
        return ap, am

    def accel_part(self, part):
        """JT_PART_PM (long range only), JT_PART_SHORT (tree only) or JT_PART_ALL."""
        ap = np.zeros((self.n[0], 3), np.float32)
        am = np.zeros((self.n[1], 3), np.float32)
        _check(library().jt_accel_part(self._h, part, _ptr(ap), _ptr(am), JT_MEM_HOST),
               "jt_accel_part")
        return ap, am

    def accel_device(self, acc_p, acc_m):
        def dp(t):
            return None if t is None else C.c_void_p(t.data_ptr())
        _check(library().jt_accel(self._h, dp(acc_p), dp(acc_m), JT_MEM_DEVICE), "jt_accel")

    def set_screening(self, lambda_0, z=0.0):
        """Yukawa screening of opposite-sign pairs (set_lambda_0 /
        set_current_z), lambda_0 > 0.01 turns it on: the reference's screened
        walk in compatibility mode, the screened split model in accurate
        mode (Batch.set_screening)."""
        _check(library().jt_set_screening(self._h, lambda_0, z), "jt_set_screening")

    def set_counters(self, on):
        """Pair counters (a diagnostic, off by default): the near-field cell
        walk counts its pairs inside r_cut into timings()'s
        pair_interactions, at about 5 % of the walk's time."""
        _check(library().jt_set_counters(self._h, 1 if on else 0), "jt_set_counters")

    def step(self, dt, hubble=0.0, dtau_per_dt=1.0, nsteps=1):
        _check(library().jt_step(self._h, dt, hubble, dtau_per_dt, nsteps), "jt_step")

    def set_accel(self, acc_p, acc_m):
        """Load the accelerations at the current positions (host arrays) so
        that the next KDK step needs no opening force pass."""
        acc_p, acc_m = _f32(acc_p), _f32(acc_m)
        _check(library().jt_set_accel(self._h, _ptr(acc_p), _ptr(acc_m), JT_MEM_HOST), "jt_set_accel")

    def step_host(self, pos_p, vel_p, acc_p, pos_m, vel_m, acc_m, dt, hubble=0.0, dtau_per_dt=1.0):
        """One step of a host-held state, in place (jt_step_host): the six
        float32 (n, 3) C-contiguous arrays (pinned for full speed; acc_* may
        be None with the DKD integrator) are uploaded, stepped once and
        overwritten with the new state."""
        arrs = (pos_p, vel_p, acc_p, pos_m, vel_m, acc_m)
        for a in arrs:
            if a is not None and (not isinstance(a, np.ndarray) or a.dtype != np.float32
                                  or not a.flags["C_CONTIGUOUS"]):
                raise ValueError("step_host works in place on C-contiguous float32 arrays")
        _check(library().jt_step_host(self._h, *[_ptr(a) for a in arrs], dt, hubble, dtau_per_dt),
               "jt_step_host")

    def get_accel(self, out=None):
        """The stored accelerations (no force pass); out = [acc_p, acc_m]."""
        ap, am = out if out is not None else (np.zeros((self.n[0], 3), np.float32),
                                              np.zeros((self.n[1], 3), np.float32))
        _check(library().jt_get_accel(self._h, _ptr(ap), _ptr(am), JT_MEM_HOST), "jt_get_accel")
        return ap, am

    def get_state(self, out=None):
        """Positions and velocities in the caller's order; out = four
        preallocated (pinned, say) float32 arrays to fill."""
        if out is not None and not self._signed:
            _check(library().jt_get_state(self._h, *[_ptr(a) for a in out], JT_MEM_HOST), "jt_get_state")
            return tuple(out)
        if self._signed:
            pos = np.zeros((sum(self.n), 3), np.float32)
            vel = np.zeros((sum(self.n), 3), np.float32)
            _check(library().jt_get_state_signed(self._h, _ptr(pos), _ptr(vel), JT_MEM_HOST),
                   "jt_get_state_signed")
            return pos, vel
        pp = np.zeros((self.n[0], 3), np.float32)
        vp = np.zeros((self.n[0], 3), np.float32)
        pm = np.zeros((self.n[1], 3), np.float32)
        vm = np.zeros((self.n[1], 3), np.float32)
        _check(library().jt_get_state(self._h, _ptr(pp), _ptr(vp), _ptr(pm), _ptr(vm), JT_MEM_HOST),
               "jt_get_state")
        return pp, vp, pm, vm

    def debug_tree(self, species):
        n = self.n[species]
        nn = max(2 * n - 1, 1)
        morton = np.zeros(max(n, 1), np.uint32)
        perm = np.zeros(max(n, 1), np.int32)
        left = np.zeros(nn, np.int32)
        right = np.zeros(nn, np.int32)
        parent = np.zeros(nn, np.int32)
        _check(library().jt_debug_tree(self._h, species, _ptr(morton), _ptr(perm), _ptr(left),
                                       _ptr(right), _ptr(parent)), "jt_debug_tree")
        return dict(morton=morton[:n], perm=perm[:n], left=left, right=right, parent=parent)

    def checkpoint(self, path, meta=None):
        """Write the state to a snapshot_v3 file (caller order, signs)."""
        meta = meta if meta is not None else snapshot_meta()
        _check(library().jt_checkpoint(self._h, str(path).encode(), C.byref(meta)), "jt_checkpoint")

    def diagnostics(self, n_cells=32):
        """FP64 device diagnostics: segregation metrics, kinetic energy,
        momentum and mean position per species."""
        d = jt_diag()
        _check(library().jt_diagnostics(self._h, n_cells, C.byref(d)), "jt_diagnostics")
        return d.to_dict()

    def energy(self, n_sample=20000):
        """FP64 kinetic energy and sampled same-species binding energy."""
        e = jt_energy()
        _check(library().jt_energy_sampled(self._h, n_sample, C.byref(e)), "jt_energy_sampled")
        return e.to_dict()

    def virialize(self, n_sample=20000):
        """Scale velocities to 2 KE = |PE_binding|; returns alpha."""
        a = C.c_double(1.0)
        _check(library().jt_virialize_sampled(self._h, n_sample, C.byref(a)), "jt_virialize_sampled")
        return a.value

    def walk_counters(self):
        """(iterations, ranges, chunks, trips) of a -DJT_WALK_COUNT build."""
        v = (C.c_int64 * 4)()
        _check(library().jt_walk_counters(self._h, v), "jt_walk_counters")
        return tuple(v)

    def timings(self):
        t = jt_timings()
        _check(library().jt_get_timings(self._h, C.byref(t)), "jt_get_timings")
        return {k: getattr(t, k) for k, _ in jt_timings._fields_}


def walk_tuning():
    """The walk launch shapes the autotuner picked so far (text)."""
    buf = C.create_string_buffer(4096)
    _check(library().jt_walk_tuning(buf, 4096), "jt_walk_tuning")
    return buf.value.decode()


def morton_sort_static(pos_ptr, n, box_L, morton_ptr, perm_ptr, stream=None):
    """jt_morton_sort_static on device pointers (ints or None): sorted Morton
    codes and permutation with no device allocation (n <= JT_STATIC_SORT_MAX)."""
    _check(library().jt_morton_sort_static(pos_ptr, n, box_L, morton_ptr, perm_ptr, stream),
           "jt_morton_sort_static")


class Batch:
    """Many independent boxes stepped together (a jt_batch).

    Every stage of a force pass is one kernel launch over the work of all the
    boxes passed to ``forces``/``step`` (one batched cuFFT per grid size), in
    place of the reference's one-process-per-box scans.  Boxes keep their own
    Config (all accurate/KDK with the same pm_order, pm_interlace, k_min).
    """

    def __init__(self, graphs=False):
        self._b = C.c_void_p()
        _check(library().jt_batch_create(C.byref(self._b)), "jt_batch_create")
        self.boxes = {}
        if graphs:
            self.set_graphs(True)

    def set_graphs(self, on):
        """Replay each batched step as a CUDA graph (captured per set of boxes)."""
        _check(library().jt_batch_set_graphs(self._b, 1 if on else 0), "jt_batch_set_graphs")

    def set_counters(self, on):
        """Pair counters of the batch's passes (Solver.set_counters)."""
        _check(library().jt_batch_set_counters(self._b, 1 if on else 0), "jt_batch_set_counters")

    def trim(self):
        """Release the per-pass scratch pools (they regrow on the next pass)."""
        _check(library().jt_batch_trim(self._b), "jt_batch_trim")

    def close(self):
        if self._b:
            library().jt_batch_destroy(self._b)
            self._b = C.c_void_p()
            self.boxes = {}

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def estimate(config: Config, n_p, n_m):
        """(persistent, scratch) device bytes of one box; no device work."""
        cfg = config.resolved().to_c()
        a, b = C.c_size_t(), C.c_size_t()
        _check(library().jt_batch_estimate(C.byref(cfg), n_p, n_m, C.byref(a), C.byref(b)),
               "jt_batch_estimate")
        return a.value, b.value

    def add(self, config: Config, pos_p, vel_p, pos_m, vel_m):
        """Add one box (host arrays); returns its id."""
        pos_p = _f32(pos_p) if pos_p is not None else np.zeros((0, 3), np.float32)
        pos_m = _f32(pos_m) if pos_m is not None else np.zeros((0, 3), np.float32)
        vel_p = None if vel_p is None else _f32(vel_p)
        vel_m = None if vel_m is None else _f32(vel_m)
        cfg = config.resolved().to_c()
        bid = C.c_int(-1)
        _check(library().jt_batch_add(self._b, C.byref(cfg), _ptr(pos_p), _ptr(vel_p), len(pos_p),
                                      _ptr(pos_m), _ptr(vel_m), len(pos_m), JT_MEM_HOST,
                                      C.byref(bid)), "jt_batch_add")
        self.boxes[bid.value] = (len(pos_p), len(pos_m))
        return bid.value

    def checkpoint_async(self, box_id, path, meta=None):
        """Start a snapshot_v3 checkpoint of one box that overlaps the next
        step; collect it with checkpoint_wait()."""
        meta = meta if meta is not None else snapshot_meta()
        _check(library().jt_batch_checkpoint_async(self._b, box_id, str(path).encode(), C.byref(meta)),
               "jt_batch_checkpoint_async")

    def checkpoint_wait(self):
        _check(library().jt_batch_checkpoint_wait(self._b), "jt_batch_checkpoint_wait")

    def add_zeldovich(self, config: Config, n_side, seed=42, rms_frac=0.3, vel_factor=0.05):
        """Add a box whose Zel'dovich lattice ICs are generated on the device."""
        cfg = config.resolved().to_c()
        p = ics_params(n_side, config.box_L, seed, rms_frac, vel_factor)
        bid = C.c_int(-1)
        _check(library().jt_batch_add_zeldovich(self._b, C.byref(cfg), C.byref(p), C.byref(bid)),
               "jt_batch_add_zeldovich")
        self.boxes[bid.value] = (n_side ** 3, n_side ** 3)
        return bid.value

    def prepare(self, pm_grid):
        """Create every cuFFT plan a pass over boxes of this grid size can use
        (jt_batch_prepare), so that no later step makes one."""
        _check(library().jt_batch_prepare(self._b, pm_grid), "jt_batch_prepare")

    def set_screening(self, box_id, lambda_0, z=0.0):
        """Yukawa screening (kappa = 1 / (lambda_0 sqrt(1 + z))) of one box's
        opposite-species pairs in the split model; lambda_0 <= 0.01: off."""
        _check(library().jt_batch_set_screening(self._b, box_id, lambda_0, z), "jt_batch_set_screening")

    def remove(self, box_id):
        _check(library().jt_batch_remove(self._b, box_id), "jt_batch_remove")
        self.boxes.pop(box_id, None)

    @staticmethod
    def _ids(ids):
        arr = (C.c_int * len(ids))(*ids)
        return arr, len(ids)

    def forces(self, ids, part=JT_PART_ALL):
        arr, n = self._ids(ids)
        _check(library().jt_batch_forces(self._b, arr, n, part), "jt_batch_forces")

    def step(self, ids, dt, hubble=0.0, dtau_per_dt=1.0, nsteps=1):
        """nsteps KDK steps; dt/hubble/dtau_per_dt scalars or one per box."""
        arr, n = self._ids(ids)
        dts = np.broadcast_to(np.asarray(dt, np.float64), (n,))
        hs = np.broadcast_to(np.asarray(hubble, np.float64), (n,))
        ds = np.broadcast_to(np.asarray(dtau_per_dt, np.float64), (n,))
        args = (jt_step_args * n)(*[jt_step_args(float(dts[k]), float(hs[k]), float(ds[k]))
                                    for k in range(n)])
        _check(library().jt_batch_step(self._b, arr, n, args, nsteps), "jt_batch_step")

    def accel(self, box_id):
        n_p, n_m = self.boxes[box_id]
        ap = np.zeros((n_p, 3), np.float32)
        am = np.zeros((n_m, 3), np.float32)
        _check(library().jt_batch_get_accel(self._b, box_id, _ptr(ap), _ptr(am), JT_MEM_HOST),
               "jt_batch_get_accel")
        return ap, am

    def get_state(self, box_id):
        n_p, n_m = self.boxes[box_id]
        out = [np.zeros((n, 3), np.float32) for n in (n_p, n_p, n_m, n_m)]
        _check(library().jt_batch_get_state(self._b, box_id, *[_ptr(a) for a in out], JT_MEM_HOST),
               "jt_batch_get_state")
        return tuple(out)

    def diagnostics(self, box_id, n_cells=32):
        d = jt_diag()
        _check(library().jt_batch_diagnostics(self._b, box_id, n_cells, C.byref(d)),
               "jt_batch_diagnostics")
        return d.to_dict()

    def memory(self):
        a, b = C.c_size_t(), C.c_size_t()
        _check(library().jt_batch_memory(self._b, C.byref(a), C.byref(b)), "jt_batch_memory")
        return a.value, b.value

    def timings(self):
        t = jt_timings()
        _check(library().jt_batch_get_timings(self._b, C.byref(t)), "jt_batch_get_timings")
        return {k: getattr(t, k) for k, _ in jt_timings._fields_}


class Server:
    """Serving loop over a batch (a jt_server): jobs admitted by an HBM budget,
    step requests served by continuous batching, finished jobs evicted to
    pinned host memory, idle jobs swapped out to make room."""

    def __init__(self, hbm_budget_bytes):
        self._s = C.c_void_p()
        _check(library().jt_server_create(int(hbm_budget_bytes), C.byref(self._s)), "jt_server_create")
        self.jobs = {}

    def close(self):
        if self._s:
            library().jt_server_destroy(self._s)
            self._s = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def add_job(self, config: Config, pos_p, vel_p, pos_m, vel_m, steps, dt, hubble=0.0,
                dtau_per_dt=1.0):
        pos_p = _f32(pos_p) if pos_p is not None else np.zeros((0, 3), np.float32)
        pos_m = _f32(pos_m) if pos_m is not None else np.zeros((0, 3), np.float32)
        vel_p = None if vel_p is None else _f32(vel_p)
        vel_m = None if vel_m is None else _f32(vel_m)
        cfg = config.resolved().to_c()
        args = jt_step_args(float(dt), float(hubble), float(dtau_per_dt))
        jid = C.c_int(-1)
        _check(library().jt_server_add_job(self._s, C.byref(cfg), _ptr(pos_p), _ptr(vel_p), len(pos_p),
                                           _ptr(pos_m), _ptr(vel_m), len(pos_m), int(steps),
                                           C.byref(args), C.byref(jid)), "jt_server_add_job")
        self.jobs[jid.value] = (len(pos_p), len(pos_m))
        return jid.value

    @staticmethod
    def job_need(config: Config, n_p, n_m):
        """Budget bytes one job needs alone (no device work)."""
        cfg = config.resolved().to_c()
        b = C.c_size_t()
        _check(library().jt_server_job_need(C.byref(cfg), n_p, n_m, C.byref(b)), "jt_server_job_need")
        return b.value

    def request(self, job, t_arrival=-1.0):
        _check(library().jt_server_request(self._s, job, float(t_arrival)), "jt_server_request")

    def clock(self):
        return library().jt_server_clock(self._s)

    def poll(self):
        """Admit what fits and run one batched step; returns requests served."""
        n = C.c_int(0)
        _check(library().jt_server_poll(self._s, C.byref(n)), "jt_server_poll")
        return n.value

    def serve(self, t, jobs):
        """Replay arrival times t (seconds, ascending) of requests for jobs."""
        t = np.ascontiguousarray(t, np.float64)
        jobs = np.ascontiguousarray(jobs, np.int32)
        _check(library().jt_server_serve(self._s, _ptr(t), _ptr(jobs), len(t)), "jt_server_serve")

    def job_state(self, job):
        st, done = C.c_int(), C.c_int()
        _check(library().jt_server_job_state(self._s, job, C.byref(st), C.byref(done)),
               "jt_server_job_state")
        return st.value, done.value

    def get_accel(self, job):
        """(acc_p, acc_m) the job holds at its current positions."""
        n_p, n_m = self.jobs[job]
        ap, am = np.zeros((n_p, 3), np.float32), np.zeros((n_m, 3), np.float32)
        _check(library().jt_server_get_accel(self._s, job, _ptr(ap), _ptr(am)), "jt_server_get_accel")
        return ap, am

    def get_state(self, job):
        n_p, n_m = self.jobs[job]
        out = [np.zeros((n, 3), np.float32) for n in (n_p, n_p, n_m, n_m)]
        _check(library().jt_server_get_state(self._s, job, *[_ptr(a) for a in out]),
               "jt_server_get_state")
        return tuple(out)

    def stats(self):
        st = jt_serve_stats()
        _check(library().jt_server_stats(self._s, C.byref(st)), "jt_server_stats")
        return {k: getattr(st, k) for k, _ in jt_serve_stats._fields_}

    def set_counters(self, on):
        """Pair counters of the server's batched steps (Solver.set_counters)."""
        _check(library().jt_server_set_counters(self._s, 1 if on else 0), "jt_server_set_counters")

    def timings(self):
        """Stage times and counts of all batched steps so far, summed."""
        t = jt_timings()
        _check(library().jt_server_get_timings(self._s, C.byref(t)), "jt_server_get_timings")
        return {k: getattr(t, k) for k, _ in jt_timings._fields_}


# --------------------------------------------------------------------------
# The reference's call shapes
# --------------------------------------------------------------------------
class GpuNBodyTwoPass:
    """src/nbody_gpu_twopass.rs GpuNBodyTwoPass over the B200 engine.

    Defaults follow with_custom_ics (:2303-2336): theta 0.5, softening 0.1,
    pm_grid 256, k_min 0, mass_factor = G_cosmo * 0.3 * rho_crit * L^3 / N
    (:2320-2330).  Forces use the reference formulas (RCOMPAT) unless
    ``mode=JT_ACCURATE`` is passed; the step is the reference's
    drift-kick-drift (JT_DKD_REF) unless ``integrator=JT_KDK``.
    """

    def __init__(self, pos, vel, signs, box_size, mode=JT_RCOMPAT, integrator=JT_DKD_REF,
                 pm_grid=256):
        pos = _f32(pos)
        n = len(pos)
        self.box_size = float(box_size)
        self.theta = 0.5
        self.softening = 0.1
        self.pm_grid = pm_grid
        self.pm_k_min = 0
        g_cosmo, rho_crit, omega_m = 4.499e-15, 2.775e11, 0.3
        self.mass_factor = g_cosmo * omega_m * rho_crit * self.box_size ** 3 / n
        self.mode = mode
        self.integrator = integrator
        self._pos = pos
        self._vel = None if vel is None else _f32(vel)
        self._signs = np.ascontiguousarray(signs, dtype=np.int8)
        self._solver = None
        self._r_cut = None
        self._dirty_state = True
        self.lambda_0 = 0.0      # Yukawa screening length at z = 0 (off)
        self.current_z = 0.0

    @classmethod
    def with_custom_ics(cls, pos, vel, signs, box_size, **kw):
        return cls(pos, vel, signs, box_size, **kw)

    def set_theta(self, t):
        self._sync_state()
        self.theta = float(t)
        self._solver = None

    def set_softening(self, e):
        self._sync_state()
        self.softening = float(e)
        self._solver = None

    def set_mass_factor(self, mf):
        self._sync_state()
        self.mass_factor = float(mf)
        self._solver = None

    def set_pm_k_min(self, k):
        self._sync_state()
        self.pm_k_min = int(k)
        self._solver = None

    def set_lambda_0(self, lam):
        """Yukawa screening of opposite-sign pairs (:2305-2306); lambda(z) =
        lambda_0 sqrt(1 + z) at the next force evaluation."""
        self.lambda_0 = float(lam)
        if self._solver is not None:
            self._solver.set_screening(self.lambda_0, self.current_z)

    set_lambda_base = set_lambda_0   # the reference's alias (:2312)

    def set_current_z(self, z):
        self.current_z = float(z)
        if self._solver is not None:
            self._solver.set_screening(self.lambda_0, self.current_z)

    def kinetic_energy(self):
        """sum |v|^2 / 2, unit masses (:5070-5077), FP64 on the device."""
        self._ensure(self._r_cut or 4.5 * 1.25 * self.box_size / self.pm_grid)
        return self._solver.energy(1)["kinetic"]

    def potential_energy_binding_sampled(self, n_sample):
        """Sampled same-species binding energy (:5081-5181)."""
        self._ensure(self._r_cut or 4.5 * 1.25 * self.box_size / self.pm_grid)
        return self._solver.energy(n_sample)["pe_binding"]

    def virialize_sampled(self, n_sample):
        """Scale velocities so that 2 KE = |PE_binding| (:5186-5225)."""
        self._ensure(self._r_cut or 4.5 * 1.25 * self.box_size / self.pm_grid)
        return self._solver.virialize(n_sample)

    def segregation(self):
        """|COM+ - COM-| / L (:5364-5393), FP64 on the device."""
        self._ensure(self._r_cut or 4.5 * 1.25 * self.box_size / self.pm_grid)
        return self._solver.diagnostics(8)["segregation"]

    def _sync_state(self):
        if self._solver is not None:
            self._pos, self._vel = self._solver.get_state()

    def _ensure(self, r_cut):
        if self._solver is not None and self._r_cut == r_cut:
            return
        self._sync_state()
        n_p = int((self._signs > 0).sum())
        n_m = len(self._signs) - n_p
        mu = (n_m / n_p) if n_p else 1.0   # equal per-particle mass = mass_factor
        cfg = Config(box_L=self.box_size, pm_grid=self.pm_grid, theta=self.theta,
                     softening=self.softening, r_s=r_cut / 3.0, r_cut=r_cut, mu=mu,
                     G_mass_plus=self.mass_factor, k_min=self.pm_k_min, mode=self.mode,
                     integrator=self.integrator)
        self._solver = Solver(cfg)
        self._solver.set_state_signed(self._pos, self._vel, self._signs)
        if self.lambda_0 > 0.01:
            self._solver.set_screening(self.lambda_0, self.current_z)
        self._r_cut = r_cut

    def compute_forces(self, r_cut):
        """Accelerations of all particles in the with_custom_ics order."""
        self._ensure(r_cut)
        return self._solver.accel()

    def step_treepm_gpu(self, dt, r_cut, hubble, dtau_per_dt):
        self._ensure(r_cut)
        self._solver.step(dt, hubble, dtau_per_dt, 1)

    def get_particles(self):
        """(pos, vel, signs) in the with_custom_ics order."""
        self._sync_state()
        vel = self._vel if self._vel is not None else np.zeros_like(self._pos)
        return self._pos.copy(), vel.copy(), self._signs.copy()


@dataclass
class Particle:
    """src/nbody.rs Particle {pos, vel, mass, sign} (sign +1 / -1)."""
    pos: tuple
    vel: tuple = (0.0, 0.0, 0.0)
    mass: float = 1.0
    sign: int = 1


class TreePMForce:
    """src/treepm/treepm_force.rs TreePMForce over the B200 engine.

    new(r_cut, grid_size, box_size, theta, softening); r_s = r_cut / 3 and G = 1
    as in the reference (:35-49).  Each species' particles must share one mass
    (the engine stores one mass per species).  Positions in [-L/2, L/2).
    """

    def __init__(self, r_cut, grid_size, box_size, theta, softening, mode=JT_ACCURATE):
        self.r_cut = float(r_cut)
        self.r_s = self.r_cut / 3.0
        self.grid_size = int(grid_size)
        self.box_size = float(box_size)
        self.theta = float(theta)
        self.softening = float(softening)
        self.g_constant = 1.0
        self.mode = mode
        self._solver = None
        self._order = None

    def update(self, particles):
        pos = np.array([p.pos for p in particles], np.float64).reshape(-1, 3)
        sg = np.array([1 if p.sign > 0 else -1 for p in particles], np.int8)
        mass = np.array([abs(p.mass) for p in particles], np.float64)
        mp = mass[sg > 0]
        mm = mass[sg < 0]
        if (len(mp) and np.ptp(mp) > 1e-12 * mp.max()) or (len(mm) and np.ptp(mm) > 1e-12 * mm.max()):
            raise JanusError(JT_EINVAL, "TreePMForce.update: one mass per species")
        m_plus = float(mp[0]) if len(mp) else 1.0
        m_minus = float(mm[0]) if len(mm) else m_plus
        mu = (m_minus * len(mm)) / (m_plus * len(mp)) if len(mp) else m_minus / m_plus
        cfg = Config(box_L=self.box_size, pm_grid=self.grid_size, theta=self.theta,
                     softening=self.softening, r_s=self.r_s, r_cut=self.r_cut, mu=mu,
                     G_mass_plus=self.g_constant * m_plus, mode=self.mode)
        self._solver = Solver(cfg)
        self._solver.set_state_signed(pos.astype(np.float32), None, sg)

    def compute_all_forces(self, particles=None):
        if self._solver is None:
            raise JanusError(JT_ESTATE, "TreePMForce.compute_all_forces before update")
        return self._solver.accel().astype(np.float64)


def version():
    return library().jt_version().decode()


def short_cut(config):
    """The short-range cut the engine uses for this Config (r_cut, widened by
    cut_tail_ppm in accurate mode)."""
    c = config.to_c()
    v = C.c_double()
    _check(library().jt_config_short_cut(C.byref(c), C.byref(v)), "jt_config_short_cut")
    return v.value


def fp32_peak_tflops(iters=4096):
    """Measured FP32 FMA throughput of the current device."""
    v = C.c_double()
    _check(library().jt_fp32_peak(iters, C.byref(v)), "jt_fp32_peak")
    return v.value
