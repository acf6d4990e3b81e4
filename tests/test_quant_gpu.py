"""GPU parity of quantiser selection and quantisation with reconstruction against the
reference's golden fixtures and the oracle (bit-exact: integer reconstruction, identical
quantiser indices, skip flags and bit estimates)."""
import numpy as np
import pytest
import torch

from test_oracle import quant_case

pytestmark = pytest.mark.gpu


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_code_residue_golden_batched(gpu, golden):
    g = golden("quant.npz")
    comps, wants = [], []
    for k in range(4):
        w, h, depth, filt, intra, comp, lam, coeff, want = quant_case(g, k)
        comps.append({"coeff": dev(coeff), "intra": intra, "depth": depth, "lambda_": lam,
                      "band_wt": want["wt"].astype(np.float32), "band_ecf": want["ecf"], "band_ncb": want["ncb"]})
        wants.append(want)
    res = gpu.quant.code_residue(comps)
    for k, (c, r, want) in enumerate(zip(comps, res, wants)):
        np.testing.assert_array_equal(c["coeff"].cpu().numpy(), want["recon"], err_msg=f"case {k}")
        np.testing.assert_array_equal(r["skip"], want["skip"])
        np.testing.assert_array_equal(r["qidx"][r["skip"] == 0], want["qidx"][want["skip"] == 0])
        np.testing.assert_array_equal(r["bits"], want["bits"])
        np.testing.assert_array_equal(r["cb_skip"], want["cb_skip"])


@pytest.mark.parametrize("case", range(5))
def test_code_residue_vs_oracle_full_frames(gpu, oracle, case):
    from dirac_b200 import quant, synth

    w, h, depth, filt, intra, qf, cf = [(1920, 1080, 4, 6, 1, 7, 2), (1920, 1080, 4, 0, 0, 7, 2),
                                        (720, 576, 5, 2, 1, 5, 1), (1280, 720, 4, 1, 0, 3, 2),
                                        (352, 288, 4, 3, 1, 10, 2)][case]
    seq = synth.make_sequence(w, h, 2, n_rects=24, vmax=24, seed=600 + case, chroma={2: "420", 1: "422"}[cf])
    f = [synth.to_signed(p) for p in seq[0]]
    gfr = [synth.to_signed(p) for p in seq[1]]
    comps, wants = [], []
    for comp in range(3):
        pic = f[comp] if intra else np.clip(f[comp].astype(np.int32) - gfr[comp], -128, 127).astype(np.int16)
        coeff = oracle.dwt_forward(filt, depth, pic)
        ch, cw = coeff.shape
        lam = 10 ** ((12 - qf) / 2.5) / 16 * (1 if intra else 4)
        wt = quant.band_weights(filt, depth, cw, ch, comp, cf, 32.0, 1.0).astype(np.float32)
        ecf = np.full(3 * depth + 1, 0.75 if not intra else 1.0, np.float32)
        ncb = quant.code_blocks(depth, w, h)
        want = oracle.code_residue(intra, depth, coeff, lam, wt, ecf, ncb)
        comps.append({"coeff": dev(coeff), "intra": intra, "depth": depth, "lambda_": lam, "band_wt": wt,
                      "band_ecf": ecf, "band_ncb": ncb})
        wants.append(want)
    qout = [torch.zeros_like(c["coeff"]) for c in comps]
    res = gpu.quant.code_residue(comps, qout=qout)
    for comp, (c, r, want) in enumerate(zip(comps, res, wants)):
        recon, q, sk, bits, cbs, qo = want
        np.testing.assert_array_equal(c["coeff"].cpu().numpy(), recon, err_msg=f"comp {comp}")
        np.testing.assert_array_equal(r["skip"], sk)
        np.testing.assert_array_equal(r["qidx"][sk == 0], q[sk == 0])
        np.testing.assert_array_equal(r["bits"], bits)
        np.testing.assert_array_equal(r["cb_skip"], cbs)
        np.testing.assert_array_equal(qout[comp].cpu().numpy(), qo)
