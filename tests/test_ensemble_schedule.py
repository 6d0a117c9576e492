"""Host logic of the ensemble server's schedule table (no GPU): the capacity rule and
the loading of a measured table."""
import json

from pandora import ensemble


def test_pick_capacity_smallest_within_five_percent():
    # a rate that creeps up by less than 5% per doubling does not pull the capacity up
    rates = {"1": 2296.0, "2": 2320.0, "4": 2428.0, "8": 2493.0, "16": 2538.0, "32": 2556.0}
    assert ensemble.pick_capacity(rates) == 8
    assert ensemble.pick_capacity({1: 100.0, 2: 300.0, 4: 290.0}) == 2
    assert ensemble.pick_capacity({1: 5.0}) == 1


def test_loaded_table_takes_schedule_and_capacity_from_rates(tmp_path):
    table = {"32/0": {"best": 64, "xlpw": 1,
                      "rates": {"1": 10.0, "64": 11.0},
                      "rates_by_xlpw": {"1": {"1": 10.0, "64": 11.0},
                                        "4": {"1": 40.0, "2": 70.0, "4": 98.0, "8": 100.0}}}}
    src = tmp_path / "table.json"
    src.write_text(json.dumps(table))
    out = ensemble.autotune(sizes=(32,), precisions=(0,), start=str(src))
    assert out["32/0"]["xlpw"] == 4 and out["32/0"]["best"] == 4


def test_committed_table_is_complete():
    with open(ensemble.MEASURED_TABLE) as fh:
        table = json.load(fh)
    for n in ensemble.SIZES:
        for prec in (0, 1):
            entry = table[f"{n}/{prec}"]
            assert entry["best"] == ensemble.pick_capacity(entry["rates"])
