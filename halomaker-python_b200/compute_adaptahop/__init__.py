"""Drop-in replacement for the reference's f2py extension ``compute_adaptahop``.

The reference builds this module from fortran/compute_adaptahop.pyf and
imports it as ``from compute_adaptahop import neikdtree``
(src/compute_neiKDtree_mod.py:36).  This package exposes the same object with
the same five subroutines (pyf:9-67) and five module arrays (pyf:4-8), backed
by the B200 library libahop_b200.so.  Put the directory that contains this
package first on ``sys.path`` and the reference's driver runs unchanged.

Differences a caller can observe:
  * errors raise ``ahop_b200.AhopError`` instead of the Fortran's STOP, which
    terminates the whole process;
  * ``nbPes`` (OpenMP threads) is accepted and ignored;
  * ``optimize_nodes=True`` (the reference's opt-in moment path) is rejected.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ahop_b200 import _lib as L

__all__ = ["neikdtree"]


class _NeiKDtree:
    """Module object mirroring the Fortran module ``neikdtree``."""

    def __init__(self):
        self._clear()

    def _clear(self):
        self.liste_parts = None
        self.density = None
        self.nnodes = 0
        self.real_table = None
        self.integer_table = None

    # --- pyf:25-48, f90:591-641
    def sync_from_init_adaptahop(self, npart_in, nmembthresh_in, nmembers_in, omegal_in, omega_lambda_f_in,
                                 omega0_in, omega_f_in, aexp_max_in, af_in, hubble_in, h_f_in, boxsize2_in, lf_in,
                                 xlong_in, ylong_in, zlong_in, xlongs2_in, ylongs2_in, zlongs2_in, hub_pt_in,
                                 aexp_in, pos_shift_in):
        ps = np.asarray(pos_shift_in, np.float64).reshape(3)
        init = L.AhopInit(int(npart_in), int(nmembthresh_in), int(nmembers_in), float(omegal_in),
                          float(omega_lambda_f_in), float(omega0_in), float(omega_f_in), float(aexp_max_in),
                          float(af_in), float(hubble_in), float(h_f_in), float(boxsize2_in), float(lf_in),
                          float(xlong_in), float(ylong_in), float(zlong_in), float(xlongs2_in), float(ylongs2_in),
                          float(zlongs2_in), float(hub_pt_in), float(aexp_in), (C.c_double * 3)(*ps))
        L.check(L.lib().ahop_sync_from_init_adaptahop(C.byref(init)), "sync_from_init_adaptahop")

    # --- pyf:16-23, f90:576-589
    def sync_from_change_pos(self, npart_in, nusedpart_in, epsilon_in, fudgepsilon_in, xlong_in, boxsize2_in):
        L.check(L.lib().ahop_sync_from_change_pos(int(npart_in), int(nusedpart_in), float(epsilon_in),
                                                  float(fudgepsilon_in), float(xlong_in), float(boxsize2_in)),
                "sync_from_change_pos")

    # --- pyf:50-65, f90:643-678
    def sync_others(self, verbose_in, megaverbose_in, npart_in, nbpes_in, rho_threshold_in, massp_in, boxsize_in,
                    nhop_in, nvoisins_in, fudge_in, alphap_in, method_in, nlevelmax_in, optimize_nodes_in):
        o = L.AhopOthers(int(bool(verbose_in)), int(bool(megaverbose_in)), int(npart_in), int(nbpes_in),
                         float(rho_threshold_in), float(massp_in), float(boxsize_in), int(nhop_in),
                         int(nvoisins_in), float(fudge_in), float(alphap_in), str(method_in).encode()[:8],
                         int(nlevelmax_in), int(bool(optimize_nodes_in)))
        L.check(L.lib().ahop_sync_others(C.byref(o)), "sync_others")

    # --- pyf:9-12, f90:495-543
    def compute_adaptahop(self, pos_in, mass_in):
        pos = np.asarray(pos_in, dtype=np.float64)
        if pos.ndim != 2 or pos.shape[0] != 3:
            raise ValueError("pos_in should have shape (3,npart)")  # f90:509-512
        # the Fortran array pos(3,npart) is x0,y0,z0,x1,... in memory
        pos = np.asfortranarray(pos)
        mass = np.ascontiguousarray(mass_in, dtype=np.float64)
        n = pos.shape[1]
        if mass.shape[0] != n:
            raise ValueError("mass_in must have npart entries")
        self.close()  # f90:501
        L.check(L.lib().ahop_compute_adaptahop(pos.ctypes.data, mass.ctypes.data, n), "compute_adaptahop")
        out = L.AhopOutputs()
        L.check(L.lib().ahop_get_outputs(C.byref(out)), "get_outputs")
        nn = int(out.nnodes)
        self.nnodes = np.int32(nn)
        # Like f2py's module arrays these are views of library-owned (pinned)
        # memory, valid until the next compute_adaptahop; the reference copies
        # them out before calling close() (NEI:53-64).
        self.density = np.ctypeslib.as_array(C.cast(out.density, C.POINTER(C.c_double)), (n,))
        nused = int(out.nusedpart)
        self.liste_parts = np.ctypeslib.as_array(C.cast(out.liste_parts, C.POINTER(C.c_int32)), (nused,))
        if nn > 0:
            rt = np.ctypeslib.as_array(C.cast(out.real_table, C.POINTER(C.c_double)), (nn * 8,))
            it = np.ctypeslib.as_array(C.cast(out.integer_table, C.POINTER(C.c_int32)), (nn * 6,))
        else:
            rt = np.empty(0, np.float64)
            it = np.empty(0, np.int32)
        # Fortran real_table(8,nnodes) / integer_table(6,nnodes), column-major
        self.real_table = rt.reshape((8, nn), order="F")
        self.integer_table = it.reshape((6, nn), order="F")

    # --- pyf:67, f90:3227-3264
    def close(self):
        L.check(L.lib().ahop_close(), "close")
        self._clear()


neikdtree = _NeiKDtree()
