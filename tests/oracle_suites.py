"""Host-memory stand-ins for the 2D and 3D suite libraries, for CPU tests of
the multi-rank host (tealeaf_b200.decomp.DistHost) on gloo ranks: the run_*
entry points tealeaf_b200.host.Host calls, on numpy arrays, each computed by
the oracle's restatement of the reference omp3 kernel (oracle/tl_oracle.c).
Test infrastructure: they check the host's decomposition, face exchange and
rank sums, and are never a product path.
"""
import ctypes as C

import numpy as np

from oracle.oracle import OracleLib, OState
from tealeaf_b200.host import FIELD_IDS

P = C.POINTER(C.c_double)
_I, _D = C.c_int, C.c_double
_GRID = ("density0", "density", "energy0", "energy", "u", "u0", "p", "r", "mi", "w", "kx", "ky", "sd",
         "volume", "x_area", "y_area")
_EXCHANGED = ("density", "energy0", "energy", "u", "p", "sd")   # fields_to_exchange order
_TABLES = ("cg_alphas", "cg_betas", "cheby_alphas", "cheby_betas")


def _p(a):
    return a.ctypes.data_as(P)


class OracleSuite2D:
    def __init__(self):
        self.o = OracleLib()
        self.o.lib.o2_jacobi_iterate.restype = _D
        self.mem = {}   # chunk address -> {member: array}

    # -- plumbing -------------------------------------------------------------------
    def _get(self, cref):
        c = cref._obj
        return c, self.mem[C.addressof(c)]

    @staticmethod
    def _dims(c, s):
        return _I(c.x), _I(c.y), _I(s.halo_depth)

    def tl2d_get_error(self, buf, n):
        return 0

    def run_kernel_initialise(self, cref, sref):
        c, s = cref._obj, sref._obj
        m = {name: np.zeros(c.x * c.y) for name in _GRID}
        m.update(vertex_x=np.zeros(c.x + 1), vertex_y=np.zeros(c.y + 1), cell_x=np.zeros(c.x), cell_y=np.zeros(c.y))
        for name, arr in m.items():
            setattr(c, name, arr.ctypes.data)
        tables = {k: (C.c_double * max(s.max_iters, 1))() for k in _TABLES}
        for k, t in tables.items():
            setattr(c, k, C.cast(t, P))
        m["_tables"] = tables
        self.mem[C.addressof(c)] = m

    def run_kernel_finalise(self, cref, sref):
        self.mem.pop(C.addressof(cref._obj), None)

    def _field(self, m, address):
        for name in _GRID:
            if m[name].ctypes.data == address:
                return m[name]
        raise KeyError("no field at %#x" % address)

    # -- set-up ---------------------------------------------------------------------
    def run_set_chunk_data(self, cref, sref):
        c, m = self._get(cref)
        s = sref._obj
        x_min = s.grid_x_min + s.dx * c.left
        y_min = s.grid_y_min + s.dy * c.bottom
        self.o.o2_set_chunk_data(_I(c.x), _I(c.y), _I(s.halo_depth), _D(x_min), _D(y_min), _D(s.dx), _D(s.dy),
                                 _p(m["vertex_x"]), _p(m["vertex_y"]), _p(m["cell_x"]), _p(m["cell_y"]),
                                 _p(m["volume"]), _p(m["x_area"]), _p(m["y_area"]))

    def run_set_chunk_state(self, cref, sref, states):
        c, m = self._get(cref)
        n = sref._obj.num_states
        st = (OState * n)()
        for k in range(n):
            v = states[k]
            st[k] = OState(v.density, v.energy, v.x_min, v.y_min, 0.0, v.x_max, v.y_max, 0.0, v.radius, v.geometry)
        self.o.o2_set_chunk_state(_I(c.x), _I(c.y), _p(m["vertex_x"]), _p(m["vertex_y"]), _p(m["cell_x"]),
                                  _p(m["cell_y"]), _p(m["density"]), _p(m["energy0"]), _p(m["u"]), _I(n), st)

    def run_store_energy(self, cref, sref):
        _, m = self._get(cref)
        m["energy"][:] = m["energy0"]

    # -- halos ------------------------------------------------------------------------
    def run_local_halos(self, cref, sref, depth):
        c, m = self._get(cref)
        s = sref._obj
        nb = (_I * 4)(*[c.neighbours[f] for f in range(4)])
        for f, name in enumerate(_EXCHANGED):
            if s.fields_to_exchange[f]:
                self.o.o2_halo_field(_I(c.x), _I(c.y), _I(s.halo_depth), _I(depth), nb, _p(m[name]))

    def run_pack_or_unpack(self, cref, sref, depth, face, pack, field, buffer):
        """Face slabs as the suite's pack kernel lays them out: left/right as
        rows of `depth` values, bottom/top as `depth` rows of the interior."""
        c, m = self._get(cref)
        hd = sref._obj.halo_depth
        a = self._field(m, field).reshape(c.y, c.x)
        nx, ny = c.x - 2 * hd, c.y - 2 * hd
        if face in (0, 1):
            cols = (slice(hd, hd + depth) if pack else slice(hd - depth, hd)) if face == 0 else \
                   (slice(c.x - hd - depth, c.x - hd) if pack else slice(c.x - hd, c.x - hd + depth))
            view = a[hd:hd + ny, cols]
        else:
            rows = (slice(hd, hd + depth) if pack else slice(hd - depth, hd)) if face == 2 else \
                   (slice(c.y - hd - depth, c.y - hd) if pack else slice(c.y - hd, c.y - hd + depth))
            view = a[rows, hd:hd + nx]
        addr = C.cast(buffer, C.c_void_p).value
        buf = np.ctypeslib.as_array(C.cast(addr, P), shape=(view.size,)).reshape(view.shape)
        if pack:
            buf[...] = view
        else:
            view[...] = buf

    # -- solvers ----------------------------------------------------------------------
    def run_cg_init(self, cref, sref, rx, ry, rro):
        c, m = self._get(cref)
        s = sref._obj
        rro._obj.value += self.o.o2_cg_init(*self._dims(c, s), _I(s.coefficient), _D(rx), _D(ry),
                                            _p(m["density"]), _p(m["energy"]), _p(m["u"]), _p(m["p"]),
                                            _p(m["r"]), _p(m["w"]), _p(m["kx"]), _p(m["ky"]))

    def run_cg_calc_w(self, cref, sref, pw):
        c, m = self._get(cref)
        pw._obj.value += self.o.o2_cg_calc_w(*self._dims(c, sref._obj), _p(m["p"]), _p(m["w"]), _p(m["kx"]),
                                             _p(m["ky"]))

    def run_cg_calc_ur(self, cref, sref, alpha, rrn):
        c, m = self._get(cref)
        rrn._obj.value += self.o.o2_cg_calc_ur(*self._dims(c, sref._obj), _D(alpha), _p(m["u"]), _p(m["p"]),
                                               _p(m["r"]), _p(m["w"]))

    def run_cg_calc_p(self, cref, sref, beta):
        c, m = self._get(cref)
        self.o.o2_cg_calc_p(*self._dims(c, sref._obj), _D(beta), _p(m["p"]), _p(m["r"]))

    def run_cheby_init(self, cref, sref):
        c, m = self._get(cref)
        self.o.o2_cheby_init(*self._dims(c, sref._obj), _D(c.theta), _p(m["u"]), _p(m["u0"]), _p(m["p"]),
                             _p(m["r"]), _p(m["w"]), _p(m["kx"]), _p(m["ky"]))

    def run_cheby_iterate(self, cref, sref, alpha, beta):
        c, m = self._get(cref)
        self.o.o2_cheby_iterate(*self._dims(c, sref._obj), _D(alpha), _D(beta), _p(m["u"]), _p(m["u0"]),
                                _p(m["p"]), _p(m["r"]), _p(m["w"]), _p(m["kx"]), _p(m["ky"]))

    def run_ppcg_init(self, cref, sref):
        c, m = self._get(cref)
        self.o.o2_ppcg_init(*self._dims(c, sref._obj), _D(c.theta), _p(m["r"]), _p(m["sd"]))

    def run_ppcg_inner_iteration(self, cref, sref, alpha, beta):
        c, m = self._get(cref)
        self.o.o2_ppcg_inner(*self._dims(c, sref._obj), _D(alpha), _D(beta), _p(m["u"]), _p(m["r"]),
                             _p(m["kx"]), _p(m["ky"]), _p(m["sd"]))

    def run_jacobi_init(self, cref, sref, rx, ry):
        c, m = self._get(cref)
        s = sref._obj
        self.o.o2_jacobi_init(*self._dims(c, s), _I(s.coefficient), _D(rx), _D(ry), _p(m["density"]),
                              _p(m["energy"]), _p(m["u0"]), _p(m["u"]), _p(m["kx"]), _p(m["ky"]))

    def run_jacobi_iterate(self, cref, sref, error):
        c, m = self._get(cref)
        error._obj.value = self.o.o2_jacobi_iterate(*self._dims(c, sref._obj), _p(m["kx"]), _p(m["ky"]),
                                                    _p(m["u0"]), _p(m["u"]), _p(m["r"]))

    # -- solver methods and results ----------------------------------------------------
    def run_copy_u(self, cref, sref):
        c, m = self._get(cref)
        self.o.o2_copy_u(*self._dims(c, sref._obj), _p(m["u0"]), _p(m["u"]))

    def run_calculate_residual(self, cref, sref):
        c, m = self._get(cref)
        self.o.o2_calculate_residual(*self._dims(c, sref._obj), _p(m["u"]), _p(m["u0"]), _p(m["r"]),
                                     _p(m["kx"]), _p(m["ky"]))

    def run_calculate_2norm(self, cref, sref, field, norm):
        c, m = self._get(cref)
        norm._obj.value += self.o.o2_calculate_2norm(*self._dims(c, sref._obj), _p(self._field(m, field)))

    def run_finalise(self, cref, sref):
        c, m = self._get(cref)
        self.o.o2_finalise(*self._dims(c, sref._obj), _p(m["energy"]), _p(m["density"]), _p(m["u"]))

    def run_field_summary(self, cref, sref, vol, mass, ie, temp):
        c, m = self._get(cref)
        out = (C.c_double * 4)()
        self.o.o2_field_summary(*self._dims(c, sref._obj), _p(m["volume"]), _p(m["density"]),
                                _p(m["energy0"]), _p(m["u"]), out)
        for ref, v in zip((vol, mass, ie, temp), out):
            ref._obj.value += v

    def tl2d_download_field(self, cref, sref, field_id, host, count):
        _, m = self._get(cref)
        name = {v: k for k, v in FIELD_IDS.items()}[field_id]
        src = m[name]
        assert src.size == count
        C.memmove(host.value if isinstance(host, C.c_void_p) else host, src.ctypes.data, 8 * count)


# ------------------------------------------------------------------------------------ 3D --
_GRID3 = ("density0", "density", "energy0", "energy", "vec_u", "vec_u0", "vec_p", "vec_r", "vec_mi", "vec_w",
          "vec_kx", "vec_ky", "vec_kz", "vec_sd", "volume", "x_area", "y_area", "z_area")
_EXCHANGED3 = ("density", "energy0", "energy", "vec_u", "vec_p", "vec_sd")
_MEMBER3 = {"u": "vec_u", "u0": "vec_u0", "p": "vec_p", "r": "vec_r", "mi": "vec_mi", "w": "vec_w",
            "kx": "vec_kx", "ky": "vec_ky", "kz": "vec_kz", "sd": "vec_sd"}


class OracleSuite3D:
    def __init__(self):
        self.o = OracleLib()
        self.mem = {}

    def _get(self, cref):
        c = cref._obj
        return c, self.mem[C.addressof(c)]

    @staticmethod
    def _dims(c, s):
        return _I(c.x), _I(c.y), _I(c.z), _I(s.halo_depth)

    def _field(self, m, address):
        for name in _GRID3:
            if m[name].ctypes.data == address:
                return m[name]
        raise KeyError("no field at %#x" % address)

    def tl3d_get_error(self, buf, n):
        return 0

    def run_kernel_initialise(self, cref, sref):
        c, s = cref._obj, sref._obj
        m = {name: np.zeros(c.x * c.y * c.z) for name in _GRID3}
        m.update(vertex_x=np.zeros(c.x + 1), vertex_y=np.zeros(c.y + 1), vertex_z=np.zeros(c.z + 1),
                 cell_x=np.zeros(c.x), cell_y=np.zeros(c.y), cell_z=np.zeros(c.z))
        for name, arr in m.items():
            setattr(c, name, arr.ctypes.data)
        tables = {k: (C.c_double * max(s.max_iters, 1))() for k in _TABLES}
        for k, t in tables.items():
            setattr(c, k, C.cast(t, P))
        m["_tables"] = tables
        self.mem[C.addressof(c)] = m

    def run_kernel_finalise(self, cref, sref):
        self.mem.pop(C.addressof(cref._obj), None)

    def run_set_chunk_data(self, cref, sref):
        c, m = self._get(cref)
        s = sref._obj
        mins = (s.grid_x_min + s.dx * c.left, s.grid_y_min + s.dy * c.bottom, s.grid_z_min + s.dz * c.back)
        self.o.o3_set_chunk_data(*self._dims(c, s), *[_D(v) for v in mins], _D(s.dx), _D(s.dy), _D(s.dz),
                                 _p(m["vertex_x"]), _p(m["vertex_y"]), _p(m["vertex_z"]), _p(m["cell_x"]),
                                 _p(m["cell_y"]), _p(m["cell_z"]), _p(m["volume"]), _p(m["x_area"]),
                                 _p(m["y_area"]), _p(m["z_area"]))

    def run_set_chunk_state(self, cref, sref, states):
        c, m = self._get(cref)
        n = sref._obj.num_states
        st = (OState * n)()
        for k in range(n):
            v = states[k]
            st[k] = OState(v.density, v.energy, v.x_min, v.y_min, v.z_min, v.x_max, v.y_max, v.z_max, v.radius,
                           v.geometry)
        self.o.o3_set_chunk_state(_I(c.x), _I(c.y), _I(c.z), _p(m["vertex_x"]), _p(m["vertex_y"]),
                                  _p(m["vertex_z"]), _p(m["cell_x"]), _p(m["cell_y"]), _p(m["cell_z"]),
                                  _p(m["density"]), _p(m["energy0"]), _p(m["vec_u"]), _I(n), st)

    def run_store_energy(self, cref, sref):
        _, m = self._get(cref)
        m["energy"][:] = m["energy0"]

    def run_local_halos(self, cref, sref, depth):
        c, m = self._get(cref)
        s = sref._obj
        nb = (_I * 6)(*[c.neighbours[f] for f in range(6)])
        for f, name in enumerate(_EXCHANGED3):
            if s.fields_to_exchange[f]:
                self.o.o3_halo_field(*self._dims(c, s), _I(depth), nb, _p(m[name]))

    def run_pack_or_unpack(self, cref, sref, depth, face, pack, field, buffer):
        """Face slabs of `depth` layers over the interior of the other two
        axes, array order z, y, x."""
        c, m = self._get(cref)
        hd = sref._obj.halo_depth
        a = self._field(m, field).reshape(c.z, c.y, c.x)
        axis = 2 - face // 2
        n = a.shape[axis]
        sl = [slice(hd, e - hd) for e in a.shape]
        if face % 2 == 0:
            sl[axis] = slice(hd, hd + depth) if pack else slice(hd - depth, hd)
        else:
            sl[axis] = slice(n - hd - depth, n - hd) if pack else slice(n - hd, n - hd + depth)
        view = a[tuple(sl)]
        addr = C.cast(buffer, C.c_void_p).value
        buf = np.ctypeslib.as_array(C.cast(addr, P), shape=(view.size,)).reshape(view.shape)
        if pack:
            buf[...] = view
        else:
            view[...] = buf

    def run_cg_solver_init(self, cref, sref, rx, ry, rz, rro):
        c, m = self._get(cref)
        s = sref._obj
        rro._obj.value += self.o.o3_cg_init(*self._dims(c, s), _I(s.coefficient), _D(rx), _D(ry), _D(rz),
                                            _p(m["density"]), _p(m["energy"]), _p(m["vec_u"]), _p(m["vec_p"]),
                                            _p(m["vec_r"]), _p(m["vec_w"]), _p(m["vec_kx"]), _p(m["vec_ky"]),
                                            _p(m["vec_kz"]))

    def run_cg_solver_calc_w(self, cref, sref, pw):
        c, m = self._get(cref)
        pw._obj.value += self.o.o3_cg_calc_w(*self._dims(c, sref._obj), _p(m["vec_p"]), _p(m["vec_w"]),
                                             _p(m["vec_kx"]), _p(m["vec_ky"]), _p(m["vec_kz"]))

    def run_cg_solver_calc_ur(self, cref, sref, alpha, rrn):
        c, m = self._get(cref)
        rrn._obj.value += self.o.o3_cg_calc_ur(*self._dims(c, sref._obj), _D(alpha), _p(m["vec_u"]),
                                               _p(m["vec_p"]), _p(m["vec_r"]), _p(m["vec_w"]))

    def run_cg_solver_calc_p(self, cref, sref, beta):
        c, m = self._get(cref)
        self.o.o3_cg_calc_p(*self._dims(c, sref._obj), _D(beta), _p(m["vec_p"]), _p(m["vec_r"]))

    def run_cheby_solver_init(self, cref, sref):
        c, m = self._get(cref)
        self.o.o3_cheby_init(*self._dims(c, sref._obj), _D(c.theta), _p(m["vec_u"]), _p(m["vec_u0"]),
                             _p(m["vec_p"]), _p(m["vec_r"]), _p(m["vec_w"]), _p(m["vec_kx"]), _p(m["vec_ky"]),
                             _p(m["vec_kz"]))

    def run_cheby_solver_iterate(self, cref, sref, alpha, beta):
        c, m = self._get(cref)
        self.o.o3_cheby_iterate(*self._dims(c, sref._obj), _D(alpha), _D(beta), _p(m["vec_u"]),
                                _p(m["vec_u0"]), _p(m["vec_p"]), _p(m["vec_r"]), _p(m["vec_w"]),
                                _p(m["vec_kx"]), _p(m["vec_ky"]), _p(m["vec_kz"]))

    def run_ppcg_init(self, cref, sref):
        c, m = self._get(cref)
        self.o.o3_ppcg_init(*self._dims(c, sref._obj), _D(c.theta), _p(m["vec_r"]), _p(m["vec_sd"]))

    def run_ppcg_inner_iteration(self, cref, sref, alpha, beta):
        c, m = self._get(cref)
        self.o.o3_ppcg_inner(*self._dims(c, sref._obj), _D(alpha), _D(beta), _p(m["vec_u"]), _p(m["vec_r"]),
                             _p(m["vec_kx"]), _p(m["vec_ky"]), _p(m["vec_kz"]), _p(m["vec_sd"]))

    def run_jacobi_solver_init(self, cref, sref, rx, ry, rz):
        c, m = self._get(cref)
        s = sref._obj
        self.o.o3_jacobi_init(*self._dims(c, s), _I(s.coefficient), _D(rx), _D(ry), _D(rz), _p(m["density"]),
                              _p(m["energy"]), _p(m["vec_u0"]), _p(m["vec_u"]), _p(m["vec_kx"]),
                              _p(m["vec_ky"]), _p(m["vec_kz"]))

    def run_jacobi_solver_iterate(self, cref, sref, error):
        c, m = self._get(cref)
        error._obj.value = self.o.o3_jacobi_iterate(*self._dims(c, sref._obj), _p(m["vec_kx"]), _p(m["vec_ky"]),
                                                    _p(m["vec_kz"]), _p(m["vec_u0"]), _p(m["vec_u"]),
                                                    _p(m["vec_r"]))

    def run_solver_copy_u(self, cref, sref):
        c, m = self._get(cref)
        self.o.o3_copy_u(*self._dims(c, sref._obj), _p(m["vec_u0"]), _p(m["vec_u"]))

    def run_calculate_residual(self, cref, sref):
        c, m = self._get(cref)
        self.o.o3_calculate_residual(*self._dims(c, sref._obj), _p(m["vec_u"]), _p(m["vec_u0"]), _p(m["vec_r"]),
                                     _p(m["vec_kx"]), _p(m["vec_ky"]), _p(m["vec_kz"]))

    def run_calculate_2norm(self, cref, sref, field, norm):
        c, m = self._get(cref)
        norm._obj.value += self.o.o3_calculate_2norm(*self._dims(c, sref._obj), _p(self._field(m, field)))

    def run_solver_finalise(self, cref, sref):
        c, m = self._get(cref)
        self.o.o3_finalise(*self._dims(c, sref._obj), _p(m["energy"]), _p(m["density"]), _p(m["vec_u"]))

    def run_field_summary(self, cref, sref, vol, mass, ie, temp):
        c, m = self._get(cref)
        out = (C.c_double * 4)()
        self.o.o3_field_summary(*self._dims(c, sref._obj), _p(m["volume"]), _p(m["density"]),
                                _p(m["energy0"]), _p(m["vec_u"]), out)
        for ref, v in zip((vol, mass, ie, temp), out):
            ref._obj.value += v

    def tl3d_download_field(self, cref, sref, field_id, host, count):
        _, m = self._get(cref)
        name = {v: k for k, v in FIELD_IDS.items()}[field_id]
        src = m[_MEMBER3.get(name, name)]
        assert src.size == count
        C.memmove(host.value if isinstance(host, C.c_void_p) else host, src.ctypes.data, 8 * count)
