"""Roofline bookkeeping for the evaluation phases.

Algorithmic work per unit (the figures `achieved` is computed from):
* P2P   : 20 flop per body-pair interaction (the reference's convention,
          sample/barnes-hut/bh.cc:407, exafmm gpu/serial.cu:65); bound by the
          FP32 pipe (mixed) or FP64 pipe (plain).
* M2L   : 8 * sum_{j<P} (j+1)(P-j)^2 flop per translation (the reference's
          complex multiply-add count in LaplaceSphericalCPU_tapas.h:227-270);
          FP64 pipe (plain) or tensor pipe (mixed, split TF32).
* sort  : 8 LSD passes x (read + write of u64 key + u32 index) = 192 B/body;
          keys: 32 B read + 12 B written per body; HBM bound.
Peaks: HBM from MEASURED_PEAKS.json; FP32/FP64 CUDA-core peaks are nominal
(148 SMs x 128 FP32 / 64 FP64 FMA per clock x 2 x max SM clock), no measured
figure exists for them.
"""
from __future__ import annotations


# DRAM bytes of one p2p_mixed_kernel launch per body, from one ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum = 40.6 MB + 8.8 MB on a 1M-body
# unit-sphere-surface set, P=15, theta=0.4, ncrit=128).  The kernel's DRAM
# traffic is its body arrays read and results written (its source re-reads hit
# L2), so a launch's traffic is this figure times the bodies.
P2P_MIXED_DRAM_BYTES_PER_BODY = 49.4
# Same capture, m2l_tc_kernel<15>: 540.5 MB + 45.8 MB for 1.04M translations
# (the operator and multipole rows grow with P).
M2L_TC_DRAM_BYTES_PER_TRANSLATION = 565.0


def m2l_flops_per_translation(P: int) -> int:
    return 8 * sum((j + 1) * (P - j) ** 2 for j in range(P))


def nominal_tflops(kind: str, sm_mhz: float, sms: int = 148) -> float:
    lanes = {"fp32": 128, "fp64": 64}[kind]
    return sms * lanes * 2 * sm_mhz * 1e6 / 1e12


def dominant(phases: dict, lists: dict, tree: dict, P: int, peaks: dict, peak_src: str,
             precision: str = "mixed") -> dict:
    cand = {k: phases.get(k, 0.0) for k in ("bbox_keys", "sort", "tree", "p2m", "m2m",
                                            "traverse", "list_sort", "m2l_setup", "m2l_fp64",
                                            "m2l_tc", "p2p", "l2l", "l2p")}
    name = max(cand, key=cand.get)
    ms = cand[name]
    smx = float(peaks.get("sm_max_mhz", 1965.0))
    out = {"kernel": name, "ms": ms}
    if ms <= 0:
        return out
    n = tree.get("n_bodies", 0)
    if name == "m2l_tc":
        # tensor pipe: TF32 dense peak = half the measured bf16 dense peak
        ntc = lists.get("n_m2l_tc", 0)
        fl = float(m2l_flops_per_translation(P)) * ntc
        K = P * (P + 1)
        mp = ((K + 127) // 128) * 128
        kc = 32 if mp <= 256 else 16
        kp = ((K + kc - 1) // kc) * kc
        executed = float(lists.get("tc_tiles", 0)) * 128 * mp * kp * 2 * 3
        peak = float(peaks.get("bf16_tflops", 1590.0)) / 2
        ach = fl / (ms * 1e-3) / 1e12
        out.update(bound="tensor", achieved=ach, peak=peak, unit="TFLOP/s", frac=ach / peak,
                   peak_source=f"TF32 dense = bf16 {peak_src} / 2",
                   traffic=M2L_TC_DRAM_BYTES_PER_TRANSLATION * ntc,
                   traffic_source="ncu DRAM bytes per translation of a 1M-body capture, "
                                  "scaled by the translations",
                   executed_mma_tflops=executed / (ms * 1e-3) / 1e12,
                   work=f"{ntc} translations x {m2l_flops_per_translation(P)} flop "
                        f"(algorithmic); MMA executes 3 x 2 x 128 x {mp} x {kp} per tile")
        return out
    if name == "m2l_fp64":
        name = "m2l"
    if name == "p2p":
        fl = 20.0 * lists["n_p2p_interactions"]
        kind = "fp32" if precision == "mixed" else "fp64"
        peak = nominal_tflops(kind, smx)
        ach = fl / (ms * 1e-3) / 1e12
        traffic = P2P_MIXED_DRAM_BYTES_PER_BODY * n if precision == "mixed" else None
        out.update(bound=kind, achieved=ach, peak=peak, unit="TFLOP/s", frac=ach / peak,
                   peak_source=f"nominal {kind} at {smx:.0f} MHz", traffic=traffic,
                   traffic_source=("ncu DRAM bytes per body of a 1M-body capture, scaled by "
                                   "the bodies" if traffic else None),
                   work=f"{lists['n_p2p_interactions']} interactions x 20 flop")
    elif name == "m2l":
        fl = float(m2l_flops_per_translation(P)) * lists["n_m2l"]
        ach = fl / (ms * 1e-3) / 1e12
        peak = nominal_tflops("fp64", smx)
        out.update(bound="fp64", achieved=ach, peak=peak, unit="TFLOP/s", frac=ach / peak,
                   peak_source=f"nominal fp64 at {smx:.0f} MHz", traffic=None,
                   work=f"{lists['n_m2l']} translations x {m2l_flops_per_translation(P)} flop")
    else:
        per = {"sort": 192.0, "bbox_keys": 44.0 + 48.0, "tree": 16.0}.get(name)
        if per is None:
            out.update(bound="latency", note="no algorithmic byte/flop model for this phase")
            return out
        gbs = per * n / (ms * 1e-3) / 1e9
        peak = float(peaks["hbm_gbs"])
        out.update(bound="hbm", achieved=gbs, peak=peak, unit="GB/s", frac=gbs / peak,
                   peak_source=peak_src, traffic=None, work=f"{per} B/body x {n}")
    return out
