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


class _FakeBatch:
    """Stand-in for pandora.batch.Batch on the host: slots, tickets that complete at once,
    and a record of which requests each slot held (no device work)."""
    live = []

    def __init__(self, cls, capacity):
        self.cls, self.capacity = cls, capacity
        self.free = list(range(capacity))
        self.members = {}
        self.max_members = 0
        self.admitted = []
        _FakeBatch.live.append(self)

    def admit(self, p, slot=None):
        slot = self.free[0] if slot is None else slot
        self.free.remove(slot)
        self.members[slot] = p.seed_fluid
        self.admitted.append(p.seed_fluid)
        self.max_members = max(self.max_members, len(self.members))
        return slot

    def step(self, n=1):
        return 0

    def done(self, ticket):
        return True

    def finish(self, slot):
        self.members.pop(slot)
        return 0

    def reuse(self, slot):
        self.free.append(slot)

    def result_stats(self, slot):
        return [0.0], 0.0, 0.0

    def sync(self):
        pass

    def close(self):
        pass


def test_server_admits_in_arrival_order_within_capacity(monkeypatch):
    monkeypatch.setattr(ensemble, "Batch", _FakeBatch)
    _FakeBatch.live = []
    trace = ensemble.make_trace(60, seed=3, rate=None, steps=20, sizes=(32, 48, 64))
    caps = {f"{n}/{p}": {"best": 2, "xlpw": 0} for n in (32, 48, 64) for p in (0, 1)}
    srv = ensemble.Server(1 << 40, caps)
    res = srv.run(trace, realtime=False)
    srv.close()
    assert res["requests"] == len(trace)
    assert all(r.done is not None and r.admitted is not None for r in trace)
    by_class = {}
    for r in sorted(trace, key=lambda r: (r.arrival, r.rid)):
        by_class.setdefault(r.key, []).append(r.params.seed_fluid)
    admitted = {}
    for b in _FakeBatch.live:
        assert b.max_members <= b.capacity
        admitted.setdefault(ensemble.class_key(b.cls), []).extend(b.admitted)
    for key, seeds in by_class.items():   # every request once, first come first served in its class
        assert admitted[key] == seeds


def test_server_keeps_batches_within_budget(monkeypatch):
    monkeypatch.setattr(ensemble, "Batch", _FakeBatch)
    _FakeBatch.live = []
    trace = ensemble.make_trace(40, seed=5, rate=None, steps=10, sizes=(32, 48))
    caps = {f"{n}/{p}": {"best": 4, "xlpw": 0} for n in (32, 48) for p in (0, 1)}
    big = max(ensemble.batch_bytes(r.params, 4) for r in trace)
    srv = ensemble.Server(big + 1, caps)   # room for one batch at a time
    res = srv.run(trace, realtime=False)
    srv.close()
    assert res["requests"] == len(trace) and all(r.done is not None for r in trace)
    assert res["peak_batch_bytes"] <= big + 1
    assert len(_FakeBatch.live) > 4      # classes took turns, idle batches closed for others
