"""Per-map accuracy of one set of maps against a reference set (device tensors).

The error of a pixel is |got - ref| / max(|ref|, RMS(ref)): a relative error where the map
is large and an error relative to the map's typical size where it passes through zero.
Pixels with |mu| above `mu_cut` (close to a critical curve, where the magnification is
ill-conditioned) are reported on their own; the RMS is taken over the other finite pixels
(over all of them it would be dominated by the largest |mu| and loosen every bound).
"""
from __future__ import annotations


def map_errors(got: dict, ref: dict, mu_key: str = "mu", mu_cut: float = 100.0) -> dict:
    """{map: {"max", "rms", "pixels", "max_mu_gt_cut", "rms_mu_gt_cut", "pixels_mu_gt_cut"}}
    for every key of `ref` present in `got`; tensors of equal shape on one device."""
    import torch
    mu = ref.get(mu_key)
    out = {}
    for k, r in ref.items():
        if k not in got:
            continue
        g = got[k]
        fin = torch.isfinite(r)
        high = (torch.abs(mu) > mu_cut) & torch.isfinite(mu) if mu is not None else torch.zeros_like(fin)
        low = fin & ~high
        rl = r[low]
        rms = float(torch.sqrt(torch.mean(rl * rl))) if rl.numel() else 0.0
        den = torch.clamp(torch.abs(r), min=rms)
        den = torch.where(den > 0, den, torch.ones_like(den))
        e = torch.abs(g - r) / den  # NaN where got is not finite: the max is then NaN
        row = {}
        for label, m in (("", low), ("_mu_gt_cut", fin & high)):
            n = int(m.sum())
            em = e[m]
            row["max" + label] = float(torch.nan_to_num(em, nan=float("inf")).max()) if n else 0.0
            row["rms" + label] = float(torch.sqrt(torch.mean(em * em))) if n else 0.0
            row["pixels" + label] = n
        out[k] = row
    return out
