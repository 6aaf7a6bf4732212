"""Host side of the OpenPBR boundary (no GPU): the C ABI descriptor layout and
defaults, and the oracle's packing of the same record."""
import ctypes as C

import numpy as np

import oracle as orc
import tpt


def test_defaults_match_openpbr_material_new():
    d = tpt.OpenPbrDesc()
    tpt.lib().tpt_openpbr_defaults(C.byref(d))
    assert bytes(d) == bytes(tpt.openpbr_desc({}))
    assert bytes(d) == orc.pack_openpbr({}).tobytes()


def test_descriptor_bytes_agree_with_oracle_packing():
    rng = np.random.default_rng(5)
    for _ in range(20):
        m = {}
        for name, k, _ in tpt.OPENPBR_FIELDS:
            if name == "geometry_thin_walled" or rng.random() < 0.5:
                continue
            m[name] = rng.random(3).astype(np.float32) if k == 3 else np.float32(rng.random() * 2)
        assert bytes(tpt.openpbr_desc(m)) == orc.pack_openpbr(m).tobytes()


def test_field_offsets_follow_the_header():
    names = [n for n, _, _ in tpt.OPENPBR_FIELDS]
    assert names[0] == "base_weight" and names[-1] == "transmission_dispersion_abbe_number"
    assert tpt.OpenPbrDesc.base_color.offset == 4
    assert tpt.OpenPbrDesc.geometry_thin_walled.offset == 42 * 4
    assert tpt.OpenPbrDesc.transmission_dispersion_scale.offset == 43 * 4
    assert tpt.OpenPbrDesc.transmission_dispersion_abbe_number.offset == 44 * 4
