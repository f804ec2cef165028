"""Host logic of StreamOrder (the cross-stream order of cached plans and
scans), with stand-ins for CUDA streams and events: no GPU.

A use on the stream of the last use waits for nothing; a use from another
stream waits for an event recorded on the last stream at the switch; inside a
graph capture nothing waits; if the last stream cannot take an event any more,
the switch falls back to a device-wide synchronisation.
"""
import pytest

torch = pytest.importorskip("torch")
from wideanglepropagation_b200 import propagation as P  # noqa: E402


class FakeEvent:
    log = []

    def record(self, stream):
        if stream.dead:
            raise RuntimeError("invalid resource handle")
        FakeEvent.log.append(("record", stream.cuda_stream))
        self.on = stream.cuda_stream


class FakeStream:
    def __init__(self, handle, dead=False):
        self.cuda_stream, self.dead, self.device = handle, dead, "cuda:0"

    def wait_event(self, ev):
        FakeEvent.log.append(("wait", self.cuda_stream, ev.on))


@pytest.fixture
def fake_cuda(monkeypatch):
    FakeEvent.log = []
    state = {"capturing": False, "synced": 0}
    monkeypatch.setattr(torch.cuda, "Event", FakeEvent)
    monkeypatch.setattr(torch.cuda, "is_current_stream_capturing", lambda: state["capturing"])

    def sync(device=None):
        state["synced"] += 1
    monkeypatch.setattr(torch.cuda, "synchronize", sync)
    return state


def test_same_stream_costs_nothing(fake_cuda):
    o, s1 = P.StreamOrder(), FakeStream(1)
    for _ in range(3):
        assert o.begin(s1) is s1
        o.end(s1)
    assert FakeEvent.log == []


def test_switch_waits_for_the_last_stream(fake_cuda):
    o, s1, s2 = P.StreamOrder(), FakeStream(1), FakeStream(2)
    o.begin(s1)
    o.end(s1)
    o.begin(s2)
    o.end(s2)
    assert FakeEvent.log == [("record", 1), ("wait", 2, 1)]
    FakeEvent.log.clear()
    o.begin(s2)                 # back on the stream of the last use: nothing
    o.end(s2)
    o.begin(s1)                 # and a switch back waits for stream 2
    assert FakeEvent.log == [("record", 2), ("wait", 1, 2)]


def test_first_use_waits_for_nothing(fake_cuda):
    o = P.StreamOrder()
    o.begin(FakeStream(7))
    assert FakeEvent.log == []


def test_capture_neither_waits_nor_blocks_later_switches(fake_cuda):
    o, s1, cap, s3 = P.StreamOrder(), FakeStream(1), FakeStream(2), FakeStream(3)
    o.begin(s1)
    o.end(s1)
    fake_cuda["capturing"] = True
    o.begin(cap)                # captured use: no dependency across the capture boundary
    o.end(cap)
    assert FakeEvent.log == []
    fake_cuda["capturing"] = False
    o.begin(s3)                 # eager use after the capture: waits for the capture's stream
    assert FakeEvent.log == [("record", 2), ("wait", 3, 2)]


def test_dead_last_stream_falls_back_to_device_sync(fake_cuda):
    o, gone, s2 = P.StreamOrder(), FakeStream(1, dead=True), FakeStream(2)
    o.begin(gone)
    o.end(gone)
    o.begin(s2)
    assert fake_cuda["synced"] == 1
    assert FakeEvent.log == []
