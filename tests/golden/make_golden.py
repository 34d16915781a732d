"""Generate tests/golden/ref_cpu.npz from the reference's own CPU functions.

Runs ``oracle/_ref/libemc_ref.so`` -- the reference's emc.c compiled from its
source by ``make -C oracle ref`` (needs the reference checkout, so this runs in
the development container only; the .npz it writes is committed and is what
the tests read).  Every input is seeded and stored beside the output it
produced.

Functions exercised (FilipeMaia/emc file:line):
  generate_rotation_list      emc.c:49-363
  calculate_coordinates       emc.c:365-393
  get_pixel_from_voxel        emc.c:396-417
  get_slice                   emc.c:443-489
  insert_slice                emc.c:491-539
  update_slice                emc.c:541-555
  slice_weighting             emc.c:557-571
  calculate_responsability_absolute emc.c:667-682

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF_SO = os.path.join(REPO, "oracle", "_ref", "libemc_ref.so")

real = C.c_float


class Quaternion(C.Structure):
    _fields_ = [("q", real * 4)]


class Setup(C.Structure):
    _fields_ = [("side", C.c_int), ("wavelength", real), ("pixel_size", real),
                ("detector_size", C.c_int), ("detector_distance", real)]


class SpMatrix(C.Structure):
    _fields_ = [("rows", C.c_uint), ("cols", C.c_uint), ("data", C.POINTER(real))]


class SpIMatrix(C.Structure):
    _fields_ = [("rows", C.c_uint), ("cols", C.c_uint), ("data", C.POINTER(C.c_int))]


class Sp3Matrix(C.Structure):
    _fields_ = [("x", C.c_uint), ("y", C.c_uint), ("z", C.c_uint), ("data", C.POINTER(real))]


def _mat(a, side):
    a = np.ascontiguousarray(a, np.float32)
    return SpMatrix(side, side, a.ctypes.data_as(C.POINTER(real))), a


def _imat(a, side):
    a = np.ascontiguousarray(a, np.int32)
    return SpIMatrix(side, side, a.ctypes.data_as(C.POINTER(C.c_int))), a


def _3mat(a, side):
    a = np.ascontiguousarray(a, np.float32)
    return Sp3Matrix(side, side, side, a.ctypes.data_as(C.POINTER(real))), a


def load_ref():
    if not os.path.isfile(REF_SO):
        subprocess.run(["make", "-s", "-C", os.path.join(REPO, "oracle"), "ref"], check=True)
    L = C.CDLL(REF_SO)
    L.generate_rotation_list.restype = C.c_int
    L.generate_rotation_list.argtypes = [C.c_int, C.POINTER(C.POINTER(C.POINTER(Quaternion))),
                                         C.POINTER(C.POINTER(real))]
    L.calculate_coordinates.argtypes = [Setup, C.POINTER(SpMatrix), C.POINTER(SpMatrix),
                                        C.POINTER(SpMatrix)]
    L.get_slice.argtypes = [C.POINTER(Sp3Matrix), C.POINTER(SpMatrix), C.POINTER(Quaternion),
                            C.POINTER(SpMatrix), C.POINTER(SpMatrix), C.POINTER(SpMatrix)]
    L.insert_slice.argtypes = [C.POINTER(Sp3Matrix), C.POINTER(Sp3Matrix), C.POINTER(SpMatrix),
                               C.POINTER(SpIMatrix), real, C.POINTER(Quaternion),
                               C.POINTER(SpMatrix), C.POINTER(SpMatrix), C.POINTER(SpMatrix)]
    L.update_slice.restype = real
    L.update_slice.argtypes = [C.POINTER(C.POINTER(SpMatrix)), C.POINTER(C.POINTER(SpMatrix)),
                               C.POINTER(SpIMatrix), C.POINTER(real), C.POINTER(real), C.c_int,
                               C.c_int, C.c_int]
    L.slice_weighting.restype = real
    L.slice_weighting.argtypes = [C.POINTER(C.POINTER(SpMatrix)), C.POINTER(C.POINTER(SpMatrix)),
                                  C.POINTER(SpIMatrix), C.POINTER(real), C.POINTER(real), C.c_int,
                                  C.c_int, C.c_int, C.c_int]
    L.calculate_responsability_absolute.restype = real
    L.calculate_responsability_absolute.argtypes = [C.POINTER(SpMatrix), C.POINTER(SpMatrix),
                                                    C.POINTER(SpIMatrix), real, real]
    L.get_pixel_from_voxel.argtypes = [real, real, real, C.c_int, C.c_int, C.POINTER(real),
                                       C.POINTER(real)]
    return L


def ref_rotations(L, n):
    lst = C.POINTER(C.POINTER(Quaternion))()
    w = C.POINTER(real)()
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as td:  # it writes debug_*.data into the cwd
        os.chdir(td)
        try:
            R = L.generate_rotation_list(n, C.byref(lst), C.byref(w))
        finally:
            os.chdir(cwd)
    q = np.array([[lst[i].contents.q[k] for k in range(4)] for i in range(R)], np.float32)
    wt = np.array([w[i] for i in range(R)], np.float32)
    return q, wt


def ref_coordinates(L, side, wavelength, pixel_size, distance):
    setup = Setup(side, wavelength, pixel_size, 512, distance)
    mats = [_mat(np.zeros(side * side), side) for _ in range(3)]
    L.calculate_coordinates(setup, *[C.byref(m[0]) for m in mats])
    return [m[1] for m in mats]


def main():
    L = load_ref()
    rng = np.random.default_rng(20240601)
    out = {}

    # rotations (unhalved, exactly as the reference produces them)
    for n in (2, 4):
        q, w = ref_rotations(L, n)
        out[f"rot{n}_q"], out[f"rot{n}_w"] = q, w

    # detector coordinates: the reference's own setup and a strongly curved one
    setups = {"refsetup": (32, 5.6e-9, 16e-6, 0.15), "curved": (16, 1e-10, 0.02, 1.0)}
    for name, (side, wl, px, d) in setups.items():
        x, y, z = ref_coordinates(L, side, wl, px, d)
        out[f"coord_{name}"] = np.stack([x, y, z])
        out[f"coord_{name}_setup"] = np.array([side, wl, px, d], np.float64)

    # pixel-from-voxel round trip (emc.c:419-441) on the reference setup
    side, wl, px, d = setups["refsetup"]
    x, y, z = out["coord_refsetup"]
    pix = []
    for i in range(side * side):
        vox = (real * 3)(np.rint(x[i]), np.rint(y[i]), np.rint(z[i]))
        p = (real * 2)()
        L.get_pixel_from_voxel(d, wl, px, side, side, vox, p)
        pix.append((p[0], p[1]))
    out["pixel_from_voxel"] = np.array(pix, np.float32)

    # get_slice / insert_slice on a 16^3 model with the curved geometry
    side = 16
    cx, cy, cz = out["coord_curved"]
    xm, ym, zm = (_mat(a, side) for a in (cx, cy, cz))
    model = rng.uniform(0.0, 1.0, side ** 3).astype(np.float32)
    q2, _ = out["rot2_q"], None
    pick = rng.choice(len(q2), 23, replace=False)
    rots = np.concatenate([np.array([[1, 0, 0, 0]], np.float32), q2[pick]])
    out["slice_model"], out["slice_rot"] = model, rots
    m3 = _3mat(model, side)
    slices = []
    for r in rots:
        qq = Quaternion((real * 4)(*r))
        s = _mat(np.zeros(side * side), side)
        L.get_slice(C.byref(m3[0]), C.byref(s[0]), C.byref(qq), C.byref(xm[0]), C.byref(ym[0]),
                    C.byref(zm[0]))
        slices.append(s[1].copy())
    out["slice_out"] = np.array(slices, np.float32)

    mask = (rng.uniform(size=side * side) > 0.15).astype(np.int32)
    mask[rng.choice(side * side, 10, replace=False)] = 2  # counted by LL, skipped by insert
    ins_vals = rng.uniform(0.5, 2.0, (len(rots), side * side)).astype(np.float32)
    ins_w = rng.uniform(0.1, 1.0, len(rots)).astype(np.float32)
    mod_acc = _3mat(np.zeros(side ** 3), side)
    wgt_acc = _3mat(np.zeros(side ** 3), side)
    mk = _imat(mask, side)
    for r, vals, w in zip(rots, ins_vals, ins_w):
        qq = Quaternion((real * 4)(*r))
        s = _mat(vals, side)
        L.insert_slice(C.byref(mod_acc[0]), C.byref(wgt_acc[0]), C.byref(s[0]), C.byref(mk[0]),
                       float(w), C.byref(qq), C.byref(xm[0]), C.byref(ym[0]), C.byref(zm[0]))
    out["insert_mask"], out["insert_vals"], out["insert_w"] = mask, ins_vals, ins_w
    out["insert_model"], out["insert_weight"] = mod_acc[1].copy(), wgt_acc[1].copy()

    # likelihood, slice_weighting, update_slice on 6 slices x 5 images
    NS, NI = 6, 5
    sl = rng.uniform(0.0, 3.0, (NS, side * side)).astype(np.float32)
    im = rng.poisson(2.0, (NI, side * side)).astype(np.float32)
    sc = rng.uniform(0.5, 2.0, NI).astype(np.float32)
    resp = rng.uniform(0.0, 1.0, (NS, NI)).astype(np.float32)
    resp /= resp.sum(0, keepdims=True)
    sigma = 0.4
    slm = [_mat(a, side) for a in sl]
    imm = [_mat(a, side) for a in im]
    ll = np.zeros((NS, NI), np.float32)
    for r in range(NS):
        for p in range(NI):
            ll[r, p] = L.calculate_responsability_absolute(
                C.byref(slm[r][0]), C.byref(imm[p][0]), C.byref(mk[0]), sigma, float(sc[p]))
    sl_ptrs = (C.POINTER(SpMatrix) * NS)(*[C.pointer(m[0]) for m in slm])
    im_ptrs = (C.POINTER(SpMatrix) * NI)(*[C.pointer(m[0]) for m in imm])
    resp_c = np.ascontiguousarray(resp.reshape(-1))
    sc_c = np.ascontiguousarray(sc)
    rp = resp_c.ctypes.data_as(C.POINTER(real))
    sp = sc_c.ctypes.data_as(C.POINTER(real))
    wpow = np.array([L.slice_weighting(im_ptrs, sl_ptrs, C.byref(mk[0]), rp, sp, NS, side * side,
                                       p, NI) for p in range(NI)], np.float32)
    upd = [_mat(np.zeros(side * side), side) for _ in range(NS)]
    upd_ptrs = (C.POINTER(SpMatrix) * NS)(*[C.pointer(m[0]) for m in upd])
    tot = np.array([L.update_slice(im_ptrs, upd_ptrs, C.byref(mk[0]), rp, sp, NI, side * side, r)
                    for r in range(NS)], np.float32)
    out.update(ll_slices=sl, ll_images=im, ll_scaling=sc, ll_resp=resp, ll_sigma=np.float32(sigma),
               ll_out=ll, sw_out=wpow, us_slices=np.array([m[1] for m in upd], np.float32),
               us_total=tot)

    path = os.path.join(HERE, "ref_cpu.npz")
    np.savez_compressed(path, **out)
    print(f"wrote {path} ({os.path.getsize(path)} bytes, {len(out)} arrays)")


if __name__ == "__main__":
    sys.exit(main())
