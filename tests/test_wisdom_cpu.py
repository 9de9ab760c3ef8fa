"""Tuning wisdom files (cdns_wisdom_export / cdns_wisdom_import): host-only
calls, so they run without a GPU.  The format is the JSON the library writes;
malformed files are rejected without changing the cache."""
import json

import pytest

import cdns

ENTRY = '{"key": "NVIDIA B200/148|196,192,196|64,126,64", "ztl": 13, "yform": 2}'


def test_wisdom_round_trip(tmp_path):
    cdns.wisdom_forget()
    src = tmp_path / "in.json"
    src.write_text('{"cdns_wisdom": 1, "entries": [' + ENTRY +
                   ', {"key": "NVIDIA B200/148|48,48,48|16,30,16", "ztl": 0, "yform": 0, "xrw": 2}]}\n')
    cdns.wisdom_import(str(src))
    out = tmp_path / "out.json"
    cdns.wisdom_export(str(out))
    got = json.loads(out.read_text())
    assert got["cdns_wisdom"] == 1
    entries = {e["key"]: (e["ztl"], e["yform"], e["xrw"]) for e in got["entries"]}
    # an entry without "xrw" (written before that choice existed) reads as 0
    assert entries == {"NVIDIA B200/148|196,192,196|64,126,64": (13, 2, 0),
                       "NVIDIA B200/148|48,48,48|16,30,16": (0, 0, 2)}
    cdns.wisdom_forget()
    cdns.wisdom_export(str(out))
    assert json.loads(out.read_text())["entries"] == []


@pytest.mark.parametrize("text", ['{"entries": []}',
                                  '{"cdns_wisdom": 1, "entries": [{"key": "k", "ztl": 5, "yform": 0}]}',
                                  '{"cdns_wisdom": 1, "entries": [{"key": "k", "ztl": 12, "yform": 7}]}',
                                  '{"cdns_wisdom": 1, "entries": [{"key": "k", "ztl": 12, "yform": 1, "xrw": 6}]}'])
def test_wisdom_rejects_malformed(tmp_path, text):
    cdns.wisdom_forget()
    bad = tmp_path / "bad.json"
    bad.write_text(text)
    with pytest.raises(cdns.CdnsError):
        cdns.wisdom_import(str(bad))
    out = tmp_path / "out.json"
    cdns.wisdom_export(str(out))
    assert json.loads(out.read_text())["entries"] == []
