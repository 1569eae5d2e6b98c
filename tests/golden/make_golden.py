"""Generates the golden fixtures in this directory from the reference's own
code, compiled unmodified into oracle/_ref (make -C oracle ref).  Run in the
build container, where the reference sources exist:

    python tests/golden/make_golden.py

Fixtures (all produced by the reference, none hand-written):
  mie_reference_table.npz  miepdf / miecdf of src/KernelSampler.cpp:8-141
  sky_states.json          arhosek_rgb_skymodelstate_alloc_init results for the
                           configurations' (turbidity, albedo, elevation)
  sky_states_by_degree.json the same for turbidity 3, ground albedo 0.3 and a
                           sun at every whole degree of elevation 5..80
                           (azimuth 30): the batched workload's suns
                           (`python tests/golden/make_golden.py sky` writes
                           this file alone)
  c0_octree.npz            the config-0 scene (64^3 puff, seed 1) as built by the
                           C restatement of the scene build (oracle/port), which
                           the product builder must reproduce bit for bit
  ref_leaf_sequences.npz   leaf sequences of 512 rays through c0_octree from the
                           reference's step traverser (src/KernelOctree.cpp)
  ref_samplers.npz         reference Mie evaluate/sample, sun sample and brick
                           lookups (SampleVoxelSpace) on fixed inputs
  ref_c0_images.npz        two independent reference renders of config 0 at
                           128x128, 65536 spp (sums), for the image parity gate
  ref_c0_converged_256.npz the converged config-0 frame (256x256) for the
                           seconds-to-1%-RMSE measurement: the mean R of two
                           independent 32768-spp reference renders A and B,
                           as (sun + sky) rgb per sample, and their noise
                           MSE(A, B) / 4 (`python tests/golden/make_golden.py
                           c0conv` writes this file alone)
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "droplet-render_b200"))

from oracle import Port, Reference  # noqa: E402
from droplet_b200 import camera as cam  # noqa: E402
from droplet_b200 import workloads as W  # noqa: E402


def c0_config(ref: Reference, w: int, h: int, pdf, cdf) -> dict:
    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"])
    el = ref.solar_elevation(sd)
    cfgs, rads = ref.sky_state(W.SKY["turbidity"], W.SKY["albedo"], el)
    eye = cam.orbit_eye(W.CENTER, W.CAMERA["distance"], W.CAMERA["azimuth"], W.CAMERA["elevation"])
    viewi, proji = cam.camera_matrices(eye, W.CENTER, W.CAMERA["fov"], w, h)
    ss, sa, ev = W.medium("c0")
    return dict(sigma_s=ss, sigma_a=sa, scattevs=ev, sun_dir=sd, sun_color=np.asarray(W.SUN["color"], np.float32),
                sun_angle=W.SUN["angle"], turbidity=W.SKY["turbidity"], ground_albedo=W.SKY["albedo"],
                sky_configs=cfgs, sky_radiances=rads, mie_pdf=pdf, mie_cdf=cdf, viewi=viewi, proji=proji, w=w, h=h)


def sky_by_degree(ref: Reference):
    states = []
    for deg in range(5, 81):
        sd = cam.sun_direction(float(deg), W.SUN["azimuth"])
        E = ref.solar_elevation(sd)
        c, r = ref.sky_state(W.SKY["turbidity"], W.SKY["albedo"], E)
        states.append({"degree": deg, "turbidity": W.SKY["turbidity"], "albedo": W.SKY["albedo"], "elevation": E,
                       "configs": c.tolist(), "radiances": r.tolist()})
    with open(os.path.join(HERE, "sky_states_by_degree.json"), "w") as f:
        json.dump(states, f)


def c0_converged(ref: Reference, spp: int = 32768):
    pdf, cdf = ref.mie_tables()
    w = h = 256
    cfg = c0_config(ref, w, h, pdf, cdf)
    z = np.load(os.path.join(HERE, "c0_octree.npz"))
    rs = ref.scene(z["nodes"].view(np.dtype([("ce", "<f4", 4), ("chn", "<u4", 8), ("volx", "<u4", 2),
                                             ("qval", "<f4", 2)])).reshape(-1), z["bricks"])
    ref.set_threads(0)
    t = time.time()
    imgs = []
    for _ in range(2):
        sun, sky = rs.render(cfg, 0, 0, w, h, spp)
        imgs.append(((sun + sky)[..., :3].astype(np.float64) / spp))
    A, B = imgs
    ok = np.isfinite(A) & np.isfinite(B)
    R = 0.5 * (A + B)
    noise = float(((A - B)[ok] ** 2).mean()) / 4.0
    print(f"c0 converged: 2 x {w}x{h}x{spp} reference renders in {time.time() - t:.1f}s, "
          f"noise rel {np.sqrt(noise / float((R[ok] ** 2).mean())):.2e}")
    np.savez_compressed(os.path.join(HERE, "ref_c0_converged_256.npz"), mean=R.astype(np.float32), finite=ok,
                        noise_mse=noise, spp=spp, w=w, h=h)


def main():
    ref, port = Reference(), Port()
    if sys.argv[1:] == ["sky"]:
        sky_by_degree(ref)
        return
    if sys.argv[1:] == ["c0conv"]:
        c0_converged(ref)
        return
    sky_by_degree(ref)
    pdf, cdf = ref.mie_tables()
    np.savez(os.path.join(HERE, "mie_reference_table.npz"), pdf=pdf, cdf=cdf)

    # sky states: the configurations' sun (30 deg) and a sweep of elevations
    states = []
    sd = cam.sun_direction(W.SUN["elevation"], W.SUN["azimuth"])
    cases = [(W.SKY["turbidity"], W.SKY["albedo"], ref.solar_elevation(sd), "c0/c1 sun"),
             (7.0, 0.15, ref.solar_elevation(sd), "reference default T=7, albedo 0.15")]
    for deg in (5.0, 15.0, 45.0, 60.0, 80.0):
        cases.append((2.5, 0.6, float(np.radians(deg)), f"sweep {deg} deg"))
    for T, A, E, note in cases:
        c, r = ref.sky_state(T, A, E)
        states.append({"turbidity": T, "albedo": A, "elevation": E, "note": note, "configs": c.tolist(),
                       "radiances": r.tolist()})
    with open(os.path.join(HERE, "sky_states.json"), "w") as f:
        json.dump(states, f, indent=1)

    rec = W.config0_recipe(64, 1)
    org, vals = W.sparse_field(rec)
    nodes, bricks, mlevel = port.build_octree(org, vals, rec.voxel_size, 12)
    np.savez_compressed(os.path.join(HERE, "c0_octree.npz"), nodes=nodes.view(np.uint8), bricks=bricks,
                        mlevel=mlevel, block_origin=org, block_values=vals)
    rs = ref.scene(nodes, bricks)

    rng = np.random.default_rng(20261203)
    n, maxn = 512, 64
    ro = np.concatenate([rng.uniform(-1.0, 2.0, (n // 2, 3)), rng.uniform(0.15, 0.85, (n // 2, 3))]).astype(np.float32)
    rd = rng.normal(size=(n, 3))
    rd[: n // 2] = (np.asarray(W.CENTER) + rng.uniform(-0.3, 0.3, (n // 2, 3))) - ro[: n // 2]
    rd[-8:] = [[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1], [1, 1, 0], [0, 1, -1]]
    rd = (rd / np.linalg.norm(rd, axis=1, keepdims=True)).astype(np.float32)
    seq_n = np.zeros((n, maxn), np.uint32)
    seq_a = np.zeros((n, maxn), np.float32)
    seq_b = np.zeros((n, maxn), np.float32)
    cnt = np.zeros(n, np.uint32)
    for i in range(n):
        a, b, c = rs.leaf_sequence(ro[i], rd[i], full=False, maxn=maxn)
        k = len(a)
        seq_n[i, :k], seq_a[i, :k], seq_b[i, :k], cnt[i] = a, b, c, k
    np.savez_compressed(os.path.join(HERE, "ref_leaf_sequences.npz"), ro=ro, rd=rd, nodes=seq_n, tr0=seq_a, tr1=seq_b,
                        count=cnt)

    # samplers on fixed inputs
    m = 4096
    ct = np.concatenate([np.linspace(-1, 1, m // 2), rng.uniform(-1, 1, m // 2)]).astype(np.float32)
    _, mie_rgb = ref.mie_eval(ct)
    iv = rng.normal(size=(m, 3))
    iv = (iv / np.linalg.norm(iv, axis=1, keepdims=True)).astype(np.float32)
    u1 = rng.random(m).astype(np.float32)
    u2 = rng.random(m).astype(np.float32)
    mie_dir = ref.mie_sample(iv, u1, u2)
    _, _, sun_dir = ref.sun_ops(sd, np.ones(3, np.float32), W.SUN["angle"], iv, u1, u2)
    leaves = np.nonzero(nodes["volx"][:, 1] != 0xFFFFFFFF)[0]
    lid = rng.choice(leaves, m).astype(np.uint32)
    ce = nodes["ce"][lid]
    pts = (ce[:, :3] + ce[:, 3:4] * rng.uniform(-1.05, 1.05, (m, 3))).astype(np.float32)
    dens = np.array([ref.sample_voxel_space(pts[i], bricks[nodes["volx"][lid[i], 1]], ce[i]) for i in range(m)],
                    np.float32)
    np.savez_compressed(os.path.join(HERE, "ref_samplers.npz"), ct=ct, mie_rgb=mie_rgb, iv=iv, u1=u1, u2=u2,
                        mie_dir=mie_dir, sun_dir=sun_dir, leaf=lid, pts=pts, density=dens)

    # two independent reference renders of config 0 at 128x128
    w = h = 128
    spp = 65536
    cfg = c0_config(ref, w, h, pdf, cdf)
    ref.set_threads(0)
    t = time.time()
    ra = rs.render(cfg, 0, 0, w, h, spp)
    rb = rs.render(cfg, 0, 0, w, h, spp)
    print(f"reference renders: {time.time() - t:.1f}s for 2 x {w}x{h}x{spp}")
    np.savez_compressed(os.path.join(HERE, "ref_c0_images.npz"), sun_a=ra[0], sky_a=ra[1], sun_b=rb[0], sky_b=rb[1],
                        spp=spp, w=w, h=h)
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main()
