"""The HDF5 tree-brick catalogue of a snapshot (the reference's
write_tree_brick_hdf, src/input_output.py:1048-1269), assembled from the
device pipeline's rows.

The file layout is the reference's, so a merger-tree builder written for it
reads this one:
  /header   attrs: snapshot data and halo counts
  /input    attrs: the run's parameters
  /catalog/halo   one record per structure (HALO_DTYPE, ids 1..N), in the
            output units of _convert_halo_catalog_units (masses in Msun,
            positions and radii in box units, energies and L times 1e11,
            rho_0 times 100); attrs field_units (JSON) and units_version
  /member   attrs index_base = 1, layout = 'flat'; datasets index, count
            (whereIam_idxs / whereIam_counts) and pids (1-based particle ids
            grouped by structure)
The catalogue records start as the reference's clear_halo (src/halo_defs.py)
defaults; init_halos_16's tree fields (src/compute_halo_props.py:713-751)
come from the MSM selection's arrays, the property and virial fields from
the batched kernels' rows (spin from the final energies, as
compute_spin_parameter_1c runs after det_vir_1b).  Fields of the stellar,
photometric and extended-profile payloads keep their cleared values: those
payloads are not computed.

``write(f, ...)`` writes through any object with h5py's File interface;
``write_file`` opens one with h5py, which must then be installed.
"""
from __future__ import annotations

import json

import numpy as np

UNITS_VERSION = "halomaker_units_v2"
CHEM_STAR_FIELDS = tuple(f"{e}_star" for e in ("H", "O", "Fe", "Mg", "C", "N", "Si", "S", "D"))

# the record layout of the catalogue (src/halo_defs.py:302-343): a file format
HALO_DTYPE = np.dtype(
    [(f, "i4") for f in ("id", "timestep", "nmem", "ndm", "nstar", "nbsub", "hosthalo", "hostsub", "level",
                         "nextsub")]
    + [(f, "f8") for f in ("px", "py", "pz", "px*", "py*", "pz*", "vx", "vy", "vz", "Lx", "Ly", "Lz", "Lx*", "Ly*",
                           "Lz*", "sha", "shb", "shc", "m", "mdm", "m*", "r", "r*", "r50", "r90", "age", "metal")]
    + [(f, "f8") for f in CHEM_STAR_FIELDS]
    + [(f, "f8") for f in ("SFR", "SFR_r50", "SFR_r90", "SFR10", "SFR10_r50", "SFR10_r90", "spin", "sigma",
                           "sigma_dm", "sigma*", "vrot", "sig3d", "sigcyl", "vrot_r50", "sig3d_r50", "sigcyl_r50",
                           "vrot_r90", "sig3d_r90", "sigcyl_r90", "ek", "ep", "et", "rvir", "mvir", "tvir", "cvel",
                           "rho_0", "r_c", "cNFW", "cNFWerr", "vmaxcir", "rmaxcir", "inslope", "inslopeerr",
                           "mcontam")])

# unit of every catalogue field, written as the dataset's field_units attribute
_UNITS = {"int": ("id", "timestep", "hosthalo", "hostsub", "level", "nextsub"),
          "count": ("nmem", "ndm", "nstar", "nbsub"),
          "code_unit": ("px", "py", "pz", "px*", "py*", "pz*", "sha", "shb", "shc", "r", "r*", "r50", "r90", "rvir",
                        "r_c", "rmaxcir"),
          "km/s": ("vx", "vy", "vz", "sigma", "sigma_dm", "sigma*", "vrot", "sig3d", "sigcyl", "vrot_r50",
                   "sig3d_r50", "sigcyl_r50", "vrot_r90", "sig3d_r90", "sigcyl_r90", "cvel", "vmaxcir"),
          "Msun Mpc km/s": ("Lx", "Ly", "Lz", "Lx*", "Ly*", "Lz*"),
          "Msun": ("m", "mdm", "m*", "mvir", "mcontam"),
          "Gyr": ("age",), "mass_fraction": ("metal",) + CHEM_STAR_FIELDS,
          "Msun/yr": ("SFR", "SFR_r50", "SFR_r90", "SFR10", "SFR10_r50", "SFR10_r90"),
          "dimensionless": ("spin", "cNFW", "cNFWerr", "inslope", "inslopeerr"),
          "Msun (km/s)^2": ("ek", "ep", "et"), "K": ("tvir",), "Msun/kpc^3": ("rho_0",)}
CATALOG_FIELD_UNITS = {f: u for u, fs in _UNITS.items() for f in fs}

_NAN_FIELDS = ("px*", "py*", "pz*", "r*", "r50", "r90", "age", "metal") + CHEM_STAR_FIELDS + (
    "vrot", "sig3d", "sigcyl", "vrot_r50", "sig3d_r50", "sigcyl_r50", "vrot_r90", "sig3d_r90", "sigcyl_r90", "cNFW",
    "cNFWerr", "vmaxcir", "rmaxcir", "inslope", "inslopeerr")

# header and input attributes, in the order they are written; entries with a
# default are optional in ``meta`` (the reference reads them with getattr)
HEADER_ATTRS = ("npart", "nusedpart", "ndm", "nstar", "family", "massp", "aexp", "omega_t", "age_univ", "boxsize2",
                "box_comoving_mpc", "box_physical_mpc", "units_version", "hubble", "mboxp", "snapshot_dir",
                "numstep", "output_suffix", "output_tag", "output_tag_reason", "info_H0", "H_f_source",
                "nb_of_halos", "nb_of_subhalos", "createtime")
INPUT_ATTRS = ("omega_f", "omega_lambda_f", "af", "Lf", "H_f", "snapshot_dir", "numstep", "line_prefix",
               "output_suffix", "info_H0", "H_f_source", "FlagPeriod", "nMembers", "cdm", "method", "b_init",
               "nvoisins", "nhop", "rho_threshold", "fudge", "fudgepsilon", "alphap", "verbose", "megaverbose",
               "DPMMC", "SC", "dcell_min", "eps_SC", "nsteps", "dump_members", "family", "photometry")
META_DEFAULTS = {"snapshot_dir": "", "output_suffix": "", "output_tag": "", "output_tag_reason": "legacy",
                 "info_H0": np.nan, "H_f_source": "config_fallback", "line_prefix": "", "dump_members": False}


def new_catalogue(n: int) -> np.ndarray:
    """n records with clear_halo's values (src/halo_defs.py: clear_halo)."""
    cat = np.zeros(n, HALO_DTYPE)
    cat["level"] = 1
    cat["nextsub"] = -1
    for f in _NAN_FIELDS:
        cat[f] = np.nan
    return cat


def init_tree_fields(cat, level, mother, first_sister, first_daughter, numstep: int, fsub: bool = True):
    """init_halos_16 (CHP:713-751): ids, time step and the halo/subhalo tree
    fields of records 1..N (cat[k] is structure k+1) from the MSM arrays."""
    n = len(cat)
    cat["id"] = np.arange(1, n + 1)
    cat["timestep"] = numstep
    if not fsub:
        return cat
    for ih in range(1, n + 1):
        me = cat[ih - 1]
        if level[ih - 1] == 1:
            if first_daughter[ih - 1] > 0:
                me["nextsub"] = first_daughter[ih - 1]
            me["hosthalo"] = ih
            continue
        me["level"] = level[ih - 1]
        me["hostsub"] = mother[ih - 1]
        cat[me["hostsub"] - 1]["nbsub"] += 1
        if first_daughter[ih - 1] > 0:
            me["nextsub"] = first_daughter[ih - 1]
        elif first_sister[ih - 1] > 0:
            me["nextsub"] = first_sister[ih - 1]
        else:
            k = ih
            while first_sister[k - 1] <= 0 and level[k - 1] > 1:
                k = mother[k - 1]
            if level[k - 1] > 1:
                me["nextsub"] = first_sister[k - 1]
        host = cat[me["hostsub"] - 1]["hosthalo"]
        if cat[host - 1]["level"] != 1:
            raise ValueError("wrong id for halo host")
        me["hosthalo"] = host
    return cat


def fill_properties(cat, ids, counts, props, virial, gravconst: float = 430.1):
    """Property fields of the structures `ids` (1-based, with members) from
    the batched kernels' rows: props (halo_props.FIELDS) and virial
    (halo_props.VIR_FIELDS), one row per id."""
    from .halo_props import FIELDS, VIR_FIELDS
    k = np.asarray(ids, np.int64) - 1
    P = lambda f: props[:, FIELDS.index(f)]
    cat["nmem"][k] = counts
    for f in ("ndm", "nstar"):
        cat[f][k] = P(f).astype(np.int32)
    for f in ("px", "py", "pz", "vx", "vy", "vz", "Lx", "Ly", "Lz", "sha", "shb", "shc", "m", "mdm", "m*", "r",
              "sigma", "sigma_dm", "sigma*", "ek", "mcontam"):
        cat[f][k] = P(f)
    # compute_ang_mom_19 without the stellar payload (CHP:815-818)
    for f in ("Lx*", "Ly*", "Lz*"):
        cat[f][k] = np.nan
    V = lambda f: virial[:, VIR_FIELDS.index(f)]
    cat["ep"][k] = V("ep")
    cat["et"][k] = V("et")
    for f in ("rvir", "mvir", "tvir", "cvel", "rho_0", "r_c"):
        cat[f][k] = V(f)
    # compute_spin_parameter_1c (CHP:1599-1602) on the final energies
    hl = np.sqrt(cat["Lx"][k] ** 2 + cat["Ly"][k] ** 2 + cat["Lz"][k] ** 2)
    cat["spin"][k] = hl * np.sqrt(np.abs(cat["et"][k])) / cat["m"][k] ** 2.5 / gravconst
    return cat


def convert_units(cat, box_physical_mpc: float):
    """_convert_halo_catalog_units (src/input_output.py:269-289)."""
    out = cat.copy()
    for f in ("m", "mdm", "m*", "mvir", "mcontam"):
        out[f] *= 1.0e11
    for f in ("px", "py", "pz", "px*", "py*", "pz*"):
        out[f] = np.mod(out[f] / box_physical_mpc, 1.0)
    for f in ("r", "r*", "r50", "r90", "rvir", "r_c", "rmaxcir", "sha", "shb", "shc"):
        out[f] /= box_physical_mpc
    for f in ("Lx", "Ly", "Lz", "Lx*", "Ly*", "Lz*", "ek", "ep", "et"):
        out[f] *= 1.0e11
    out["rho_0"] *= 100.0
    return out


def write(f, meta: dict, cat, member_index, member_count, pids0_groupsorted):
    """Write one tree brick into the open h5py-like file `f`.  meta holds the
    header and input values by the names in HEADER_ATTRS / INPUT_ATTRS
    (aexp, boxsize2, ... as the run defines them); cat is the catalogue of
    structures 1..N before unit conversion."""
    m = dict(META_DEFAULTS)
    m.update(meta)
    m["box_comoving_mpc"] = m["boxsize2"]
    m["box_physical_mpc"] = m["aexp"] * m["boxsize2"]
    m["units_version"] = UNITS_VERSION
    header = f.create_group("header")
    for k in HEADER_ATTRS:
        header.attrs[k] = m[k]
    finput = f.create_group("input")
    for k in INPUT_ATTRS:
        finput.attrs[k] = m[k]
    out = convert_units(cat, m["aexp"] * m["boxsize2"])
    grp = f.create_group("catalog")
    ds = grp.create_dataset("halo", shape=out.shape, dtype=out.dtype, data=out, compression="lzf")
    ds.attrs["field_units"] = json.dumps(CATALOG_FIELD_UNITS, sort_keys=True)
    ds.attrs["units_version"] = UNITS_VERSION
    grp = f.create_group("member")
    grp.attrs["index_base"] = 1
    grp.attrs["layout"] = "flat"
    grp.create_dataset("index", data=member_index, compression="lzf")
    grp.create_dataset("count", data=member_count, compression="lzf")
    pids = pids0_groupsorted + 1
    chunk = min(max(1, len(pids)), 65536)
    grp.create_dataset("pids", data=pids, compression="lzf", chunks=(chunk,))


def write_file(filename: str, meta: dict, cat, member_index, member_count, pids0_groupsorted):
    """Write the tree brick to `filename` with h5py (which must be installed)."""
    try:
        import h5py
    except ImportError as e:  # not installed in every environment
        raise RuntimeError("writing a tree brick file needs h5py; ahop_b200.tree_bricks.write() takes any "
                           "object with h5py's File interface") from e
    with h5py.File(filename, "w") as f:
        write(f, meta, cat, member_index, member_count, pids0_groupsorted)


def from_snapshot(res: dict, numstep: int, gravconst: float = 430.1):
    """Catalogue and member grouping of one pipeline.run_snapshot result (run
    with particle_views=True): returns (cat, member_index, member_count,
    pids0_groupsorted) for write().  The member datasets follow the
    reference's grouping of whereIam_parts (NEI:107-119): one run per
    structure id present, unassigned particles (id 0) first; members of a
    run in increasing particle index (the reference's np.argsort is not
    stable, so its order inside a run is whatever its sort leaves)."""
    if res.get("pids_groupsorted") is None:
        raise ValueError("run the snapshot with particle_views=True for the member datasets")
    n = int(res["nstruct"])
    cat = new_catalogue(n)
    init_tree_fields(cat, res["level"], res["mother"], res["first_sister"], res["first_daughter"], numstep)
    if len(res["ids"]):
        counts = np.diff(res["offsets"]).astype(np.int32)
        fill_properties(cat, res["ids"], counts, res["props"], res["virial"], gravconst)
    return (cat, np.asarray(res["run_idxs"], np.int32), np.asarray(res["run_counts"], np.int32),
            np.asarray(res["pids_groupsorted"], np.int32))
