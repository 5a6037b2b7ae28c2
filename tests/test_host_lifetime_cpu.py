"""Host-side lifetime rules (CPU only): a context destroys the batches and
systems created on it before itself, batches before systems, whatever order
the garbage collector finalizes the Python objects in.  (The native destroy of
a system synchronizes on its context's stream, so the context must outlive it.)
"""
from molecular_simulation_code_b200 import nonbond as nb


class _FakeLib:
    def __init__(self, log):
        self.log = log

    def sofia_nb_destroy(self, handle):
        self.log.append(("ctx", handle))


class _Child:
    def __init__(self, name, log, rank=1):
        self.name, self.log, self.handle = name, log, 1
        self.close_rank = rank

    def close(self):
        if self.handle:
            self.log.append((self.name, None))
            self.handle = None


def _fake_context(log):
    c = nb.Context.__new__(nb.Context)
    c._lib = _FakeLib(log)
    c.handle = 7
    c._children = nb.weakref.WeakSet()
    return c


def test_context_closes_children_first_batches_before_systems():
    log = []
    c = _fake_context(log)
    s1, s2 = _Child("sys1", log), _Child("sys2", log)
    b = _Child("batch", log, rank=0)
    for o in (s1, b, s2):
        c.adopt(o)
    c.close()
    names = [n for n, _ in log]
    assert names[0] == "batch" and names[-1] == "ctx"
    assert sorted(names[1:3]) == ["sys1", "sys2"]
    # closing again (or a child's own finalizer) is a no-op
    c.close()
    s1.close()
    assert len(log) == 4


def test_children_are_weak_references():
    log = []
    c = _fake_context(log)
    s = _Child("sys", log)
    c.adopt(s)
    s.close()
    del s
    c.close()
    assert [n for n, _ in log] == ["sys", "ctx"]
