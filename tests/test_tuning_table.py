"""The autotuner's table (incohautocorrelate_b200/tuning/sparse_tuning.tsv),
read by every context at creation: each committed row must pass the library's
parser (a rejected row is silently skipped there), and the autotuner's writer
must produce rows that parser reads back unchanged.  CPU only."""
import os

import pytest

from incohautocorrelate_b200 import autotune

TABLE = os.path.join(os.path.dirname(autotune.__file__), "tuning", "sparse_tuning.tsv")


def parse(path):
    """The row filter of load_tuning_table (csrc/ctx.cu): mesh_edge tile_pairs
    block_threads ctas_per_sm [pairs_per_s frames cache_hints]; '#' comments."""
    rows = []
    with open(path) as fh:
        for line in fh:
            if line.startswith("#") or not line.strip():
                continue
            f = line.split()
            e, t, b, k = (int(x) for x in f[:4])
            ok = t >= 64 and 64 <= b <= 256 and b % 32 == 0 and 1 <= k <= 32
            h = int(f[6]) if len(f) >= 7 and f[6] in ("1", "2") else 2
            rows.append(dict(edge=e, tile_pairs=t, block_threads=b, ctas_per_sm=k, cache_hints=h, ok=ok))
    return rows


def test_committed_rows_are_all_accepted():
    rows = parse(TABLE)
    assert rows and all(r["ok"] for r in rows), rows
    # the two configurations the kernel is tuned on: the 65^3 small mesh and the 201^3 rotated mesh
    assert {r["edge"] for r in rows} >= {63, 199}


def test_writer_round_trips_through_the_parser(tmp_path, monkeypatch):
    monkeypatch.setattr(autotune, "TABLE", str(tmp_path / "tuning" / "sparse_tuning.tsv"))
    rows = [dict(edge=199, tile_pairs=32768, block_threads=256, ctas_per_sm=6, cache_hints=2,
                 pairs_per_s=1.87e11, frames=100000),
            dict(edge=63, tile_pairs=1024, block_threads=128, ctas_per_sm=16, cache_hints=1,
                 pairs_per_s=9.0e10, frames=100000)]
    autotune.write_table(rows)
    back = parse(autotune.TABLE)
    assert [r["edge"] for r in back] == [63, 199]  # sorted by edge
    for r in back:
        want = next(x for x in rows if x["edge"] == r["edge"])
        assert r["ok"]
        for k in ("tile_pairs", "block_threads", "ctas_per_sm", "cache_hints"):
            assert r[k] == want[k], (k, r, want)


@pytest.mark.parametrize("key,value", [("block_threads", 48), ("block_threads", 320), ("tile_pairs", 32),
                                       ("ctas_per_sm", 0), ("ctas_per_sm", 33)])
def test_parser_rejects_what_the_library_rejects(tmp_path, key, value):
    row = dict(edge=199, tile_pairs=8192, block_threads=256, ctas_per_sm=4)
    row[key] = value
    p = tmp_path / "t.tsv"
    p.write_text(f"{row['edge']}\t{row['tile_pairs']}\t{row['block_threads']}\t{row['ctas_per_sm']}\n")
    assert not parse(str(p))[0]["ok"]
