"""The CPU oracle against the reference's own known-answer constants.

Each scenario replays one reference test (same PRG seed labels and draw order);
the expected values are the reference's generated KAT constants, extracted to
tests/golden/kats.json by tests/golden/make_golden.py.
"""
import hashlib

import numpy as np
import pytest

SCENARIOS = {
    "layer3": {  # crates/via-primitives/tests/layer3_kats.rs
        "mod_switch_sym": ["MOD_SWITCH_SYM_MASK_AT_Q3", "MOD_SWITCH_SYM_BODY_AT_Q3"],
        "mod_switch_asym": ["MOD_SWITCH_ASYM_MASK_AT_Q3", "MOD_SWITCH_ASYM_BODY_AT_Q4"],
        "gen_rsk": ["GEN_RSK_J0_L0_MASK", "GEN_RSK_J0_L0_BODY", "GEN_RSK_FULL_MASK_STREAM",
                    "GEN_RSK_FULL_BODY_STREAM"],
        "ring_switch": ["RING_SWITCH_OUT_MASK", "RING_SWITCH_OUT_BODY"],
        "rekey": ["REKEY_SK_Q3_COEFFS"],
        "decrypt_asym": ["DECRYPT_ASYM_RECOVERED", "DECRYPT_ASYM_INPUT_PLAINTEXT"],
    },
    "layer4": {  # crates/via-primitives/tests/layer4_kats.rs
        "rotate": ["ROTATE_K3_MASK", "ROTATE_K3_BODY"],
        "cmux": ["CMUX_SELECT1_MASK", "CMUX_SELECT1_BODY"],
        "dmux": ["DMUX_BIT1_RESULT0_MASK", "DMUX_BIT1_RESULT0_BODY", "DMUX_BIT1_RESULT1_MASK",
                 "DMUX_BIT1_RESULT1_BODY"],
        "cmux_tree": ["CMUX_TREE_IDX3_MASK", "CMUX_TREE_IDX3_BODY"],
        "dmux_tree": [f"DMUX_TREE_IDX2_OUT{i}_{p}" for i in range(4) for p in ("MASK", "BODY")],
        "crot_forward": ["CROT_FORWARD_ROT3_MASK", "CROT_FORWARD_ROT3_BODY"],
        "crot_slot_extract": ["CROT_SLOT_EXTRACT_ROT3_MASK", "CROT_SLOT_EXTRACT_ROT3_BODY"],
        "rlwe_to_rgsw": ["RLWE_TO_RGSW_NEG_S_M_L0_MASK", "RLWE_TO_RGSW_NEG_S_M_L0_BODY",
                         "RLWE_TO_RGSW_EXT_PRODUCT_MASK", "RLWE_TO_RGSW_EXT_PRODUCT_BODY"],
        "mod_switch_rgsw": ["MOD_SWITCH_RGSW_NEG_S_M_L0_MASK", "MOD_SWITCH_RGSW_NEG_S_M_L0_BODY",
                            "MOD_SWITCH_RGSW_M_L0_MASK", "MOD_SWITCH_RGSW_M_L0_BODY"],
    },
    "layer5": {  # crates/via-primitives/tests/layer5_kats.rs
        "embed_mlwe": ["EMBED_MLWE_MASK0", "EMBED_MLWE_BODY"],
        "encrypt_lwe": ["ENCRYPT_LWE_MASKS", "ENCRYPT_LWE_BODY"],
        "conv_d": ["CONV_D_OUT_MASK0", "CONV_D_OUT_BODY"],
        "gen_lwe_to_rlwe_key": ["LWE2RLWE_KEY_STEP0_S0_L0_MASK"],
        "lwe_to_rlwe": ["LWE2RLWE_OUT_MASK", "LWE2RLWE_OUT_BODY"],
    },
    "layer6": {  # crates/via-integration/tests/layer6_kats.rs
        "encrypt_lwe_raw": ["ENCRYPT_LWE_RAW_MASKS", "ENCRYPT_LWE_RAW_BODY"],
        "gen_rlwe_to_rgsw_key": ["RLWE_TO_RGSW_KEY_S0_MASK", "RLWE_TO_RGSW_KEY_S0_BODY"],
        "query_comp": ["QUERY_COMP_MASKS", "QUERY_COMP_BODIES"],
        "resp_comp": ["RESP_COMP_MASK_Q3", "RESP_COMP_BODY_Q4"],
    },
}

CASES = [(layer, sc, name) for layer, d in SCENARIOS.items() for sc, names in d.items() for name in names]


@pytest.mark.parametrize("layer,scenario,name", CASES, ids=[f"{a}-{b}-{c}" for a, b, c in CASES])
def test_kat(oracle, golden, layer, scenario, name):
    got = oracle.kat(layer, scenario, name)
    assert list(map(int, got)) == golden[layer][name]


def test_every_golden_constant_is_checked(golden):
    checked = {(layer, name) for layer, _, name in CASES}
    for layer in ("layer3", "layer4", "layer5", "layer6"):
        for name in golden[layer]:
            assert (layer, name) in checked, f"{layer}/{name} has no replay"


@pytest.mark.parametrize("group", ["prg", "ternary", "uniform"])
def test_sampling_vectors(oracle, golden, group):
    # prim/sampling/{prg,ternary,uniform}.rs unit-test vectors.
    for name, want in golden[group].items():
        got = oracle.kat("sampling", group, name)
        assert list(map(int, got)) == [v & (2**64 - 1) for v in want], name


@pytest.mark.parametrize("n", [0, 1, 135, 136, 137, 300, 1000])
def test_shake256_matches_hashlib(oracle, n):
    for msg in (b"", b"test", bytes(range(200)), b"x" * 136):
        assert oracle.shake256(msg, n) == hashlib.shake_256(msg).digest(n)


def test_prg_stream_matches_counter_mode(oracle):
    # Shake256Prg (prg.rs:117-128): block_i = SHAKE256(seed || le64(i))[:136].
    from via_rs_b200.prg import Shake256Prg

    ref = b"".join(hashlib.shake_256(b"seed" + i.to_bytes(8, "little")).digest(136) for i in range(4))
    p = Shake256Prg(b"seed")
    assert p.bytes(500) == ref[:500]
    got = np.frombuffer(oracle.kat("sampling", "prg", "TEST_SEED_FIRST_32").astype(np.uint8).tobytes(), np.uint8)
    assert bytes(got) == Shake256Prg(b"test").bytes(32)
