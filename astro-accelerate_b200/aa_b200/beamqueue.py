"""Beams handed out to ranks at run time, with leases, through the key-value
store of torch.distributed (the TCPStore every process group has).

Beams are independent (no data moves between ranks), so the only shared
state is which beam is whose.  A rank takes the next beam with an atomic
counter, records a lease (owner and deadline) and, while it works, renews the
lease from a background thread.  When the counter runs out, a rank looks for
beams that are neither done nor under a live lease -- their owner stopped --
and takes them over with a compare-and-set on the lease, so exactly one rank
wins each takeover.  No collective is used, so ranks that stop never block
the others; the store's host (rank 0's) must stay up.

Keys under `prefix`: next (counter), lease/<i> ("<rank> <deadline>"),
done/<i> (finishing rank), ndone (counter), result/<i> (optional payload).
"""
from __future__ import annotations

import threading
import time

__all__ = ["BeamQueue"]


class BeamQueue:
    def __init__(self, store, nbeams: int, rank: int, lease_s: float = 30.0, prefix: str = "beamq"):
        self.store = store
        self.n = int(nbeams)
        self.rank = int(rank)
        self.lease_s = float(lease_s)
        self.p = prefix.rstrip("/") + "/"
        self._renew = {}
        self._lock = threading.Lock()
        self._stop = threading.Event()
        self._thread = threading.Thread(target=self._renewer, daemon=True)
        self._thread.start()

    # -- store helpers -------------------------------------------------------
    def _has(self, key: str) -> bool:
        return self.store.check([self.p + key])

    def _get(self, key: str) -> str:
        return self.store.get(self.p + key).decode()

    def _lease_value(self) -> str:
        return f"{self.rank} {time.time() + self.lease_s:.6f}"

    def _renewer(self):
        while not self._stop.wait(self.lease_s / 3.0):
            with self._lock:
                items = list(self._renew.items())
            for i, old in items:
                new = self._lease_value()
                got = self.store.compare_set(self.p + f"lease/{i}", old, new).decode()
                with self._lock:
                    if i in self._renew:
                        if got == new:
                            self._renew[i] = new
                        else:  # another rank took the beam over: stop renewing
                            del self._renew[i]

    def _hold(self, i: int, value: str):
        with self._lock:
            self._renew[i] = value

    def _release(self, i: int):
        with self._lock:
            self._renew.pop(i, None)

    # -- protocol --------------------------------------------------------------
    def done(self, i: int) -> bool:
        return self._has(f"done/{i}")

    def ndone(self) -> int:
        return int(self.store.add(self.p + "ndone", 0))

    def _finish(self, i: int, payload):
        if payload is not None:
            self.store.set(self.p + f"result/{i}", payload)
        # the first finisher marks it; a slow original owner finishing later
        # neither recounts it nor overwrites the mark
        if self.store.compare_set(self.p + f"done/{i}", "", str(self.rank)).decode() == str(self.rank):
            self.store.add(self.p + "ndone", 1)
        self._release(i)

    def _claim_next(self):
        i = int(self.store.add(self.p + "next", 1)) - 1
        if i >= self.n:
            return None
        v = self._lease_value()
        self.store.set(self.p + f"lease/{i}", v)
        self._hold(i, v)
        return i

    def _take_over(self):
        """A beam whose lease expired without it being done, or None."""
        now = time.time()
        for i in range(self.n):
            if self.done(i) or not self._has(f"lease/{i}"):
                continue
            old = self._get(f"lease/{i}")
            owner, deadline = old.split()
            if float(deadline) > now:
                continue
            new = self._lease_value()
            if self.store.compare_set(self.p + f"lease/{i}", old, new).decode() == new:
                self._hold(i, new)
                return i
        return None

    def run(self, work, poll_s: float = 0.05, timeout_s: float = 3600.0) -> list:
        """Runs work(i) -> payload (bytes/str or None) on beams until all are
        done; returns the beams this rank finished, in order."""
        mine = []
        while True:
            i = self._claim_next()
            if i is None:
                break
            self._finish(i, work(i))
            mine.append(i)
        t_end = time.time() + timeout_s
        while self.ndone() < self.n:
            if time.time() > t_end:
                raise TimeoutError(f"beam queue: {self.ndone()} of {self.n} beams done")
            i = self._take_over()
            if i is None:
                time.sleep(poll_s)
                continue
            if not self.done(i):
                self._finish(i, work(i))
                mine.append(i)
            else:
                self._release(i)
        return mine

    def result(self, i: int):
        return self.store.get(self.p + f"result/{i}") if self._has(f"result/{i}") else None

    def close(self):
        self._stop.set()
        self._thread.join(timeout=5)
