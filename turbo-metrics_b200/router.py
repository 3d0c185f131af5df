"""Multi-GPU job router over per-GPU serving replicas.

Pairs are independent, so the multi-GPU path shards jobs, not pixels: a job
(one reference + k candidates, the unit of an encoder's quality search) goes
whole to one GPU, where that GPU's `Ssim2Server` builds the reference pyramid
once and scores the candidates against it.  There is no data-path collective.

Routing policy (`RoutingPolicy`):
  * reference-cache affinity: a job whose reference id was routed before goes
    to the same GPU, which already holds that reference's pyramid (the
    cached-reference path of ssimulacra2-cuda/src/lib.rs:440-546);
  * otherwise the live GPU with the fewest outstanding bytes (host bytes of
    the images it has been given and not finished), lowest rank on a tie.

Processes (`FrontEnd`, `worker_loop`): one process per GPU, rank 0 is the
front end and also scores its own share.  Work moves in numbered steps
through a TCP store (the one the process group was initialised with): rank 0
posts each live rank's job list for step k, every rank scores its list with
its engine and posts the results; rank 0 waits for them up to a deadline.  A
rank that has not posted by the deadline -- it raised, exited or hangs -- is
dropped between steps: its affinities are forgotten and its jobs of that step
are routed again, in step k + 1, to the ranks that are left.  A rank
therefore only ever leaves between steps, with none of its work in flight on
the others, and no collective involves it after it is dropped.
"""
import pickle
import time
from dataclasses import dataclass, field
from datetime import timedelta


@dataclass
class Job:
    """One job: a reference and k candidates of one size.  `payload` is what
    the engine needs to score it (host images, or a generator spec)."""
    job_id: int
    ref_id: int
    width: int
    height: int
    n_candidates: int
    payload: object = None
    bytes_per_pixel: int = 3  # sRGB8

    @property
    def nbytes(self):
        return (1 + self.n_candidates) * self.width * self.height * self.bytes_per_pixel


@dataclass
class RoutingPolicy:
    """Reference affinity, then least outstanding bytes, over live ranks."""
    n_ranks: int
    outstanding: list = field(default_factory=list)
    alive: set = field(default_factory=set)
    affinity: dict = field(default_factory=dict)

    def __post_init__(self):
        self.outstanding = [0] * self.n_ranks
        self.alive = set(range(self.n_ranks))

    def pick(self, job):
        r = self.affinity.get(job.ref_id)
        if r is None or r not in self.alive:
            if not self.alive:
                raise RuntimeError("no live rank to route to")
            r = min(self.alive, key=lambda k: (self.outstanding[k], k))
            self.affinity[job.ref_id] = r
        self.outstanding[r] += job.nbytes
        return r

    def done(self, rank, job):
        self.outstanding[rank] -= job.nbytes

    def drop(self, rank):
        """Forget a rank that left: no more jobs, no affinities to it."""
        self.alive.discard(rank)
        self.outstanding[rank] = 0
        for ref in [k for k, v in self.affinity.items() if v == rank]:
            del self.affinity[ref]


def _key(step, what, rank=None):
    return "route/%d/%s" % (step, what) if rank is None else "route/%d/%s/%d" % (step, what, rank)


class FrontEnd:
    """Rank 0: routes jobs to the live ranks step by step and collects the
    results.  `engine` scores rank 0's own share."""

    def __init__(self, store, world, engine, deadline_s=30.0):
        self.store, self.world, self.engine = store, world, engine
        self.policy = RoutingPolicy(world)
        self.deadline_s = deadline_s
        self.step = 0
        self.placement = {}  # job_id -> rank that scored it
        self.dropped = []    # (step, rank)

    def run_step(self, jobs):
        """Route `jobs`, score them, return {job_id: scores}.  Jobs of a rank
        that misses the deadline are routed again in the next step."""
        results = {}
        pending = list(jobs)
        while pending:
            step = self.step
            self.step += 1
            lists = {r: [] for r in sorted(self.policy.alive)}
            for j in pending:
                lists[self.policy.pick(j)].append(j)
            for r, lst in lists.items():
                if r != 0:
                    self.store.set(_key(step, "jobs", r), pickle.dumps(lst))
            self.store.set(_key(step, "alive"), pickle.dumps(sorted(lists)))
            self.store.set(_key(step, "ctl"), b"jobs")
            pending = []
            if 0 in lists:  # rank 0 scores its share while the others score theirs
                for jid, sc in self.engine.score(lists[0]).items():
                    results[jid] = sc
                    self.placement[jid] = 0
                for j in lists[0]:
                    self.policy.done(0, j)
            t_end = time.monotonic() + self.deadline_s
            for r, lst in lists.items():
                if r == 0:
                    continue
                got = None
                try:
                    self.store.wait([_key(step, "res", r)], timedelta(seconds=max(0.0, t_end - time.monotonic())))
                    got = pickle.loads(self.store.get(_key(step, "res", r)))
                except Exception:  # the rank missed the deadline: it left
                    got = None
                if got is None:
                    self.policy.drop(r)
                    self.dropped.append((step, r))
                    pending.extend(lst)
                    continue
                for j in lst:
                    self.policy.done(r, j)
                for jid, sc in got.items():
                    results[jid] = sc
                    self.placement[jid] = r
        return results

    def stop(self):
        step = self.step
        self.store.set(_key(step, "alive"), pickle.dumps(sorted(self.policy.alive)))
        self.store.set(_key(step, "ctl"), b"stop")


def worker_loop(store, rank, engine, poll_s=600.0):
    """Ranks >= 1: score each step's list until rank 0 says stop (or this
    rank is no longer among the live ranks of a step).  Returns the number of
    steps it took part in."""
    step = 0
    while True:
        store.wait([_key(step, "ctl")], timedelta(seconds=poll_s))
        ctl = store.get(_key(step, "ctl"))
        alive = pickle.loads(store.get(_key(step, "alive")))
        if ctl == b"stop" or rank not in alive:
            return step
        jobs = pickle.loads(store.get(_key(step, "jobs", rank)))
        res = engine.score(jobs)
        store.set(_key(step, "res", rank), pickle.dumps(res))
        step += 1


class ServerEngine:
    """Scores jobs with this rank's GPU server (Ssim2Server on `device`):
    payload = (reference, [candidates]) host sRGB8 arrays."""

    def __init__(self, device=0, **server_kw):
        from .server import Ssim2Server
        self.server = Ssim2Server(device=device, **server_kw)

    def score(self, jobs):
        ids = [(j.job_id, self.server.submit(j.payload[0], j.payload[1])) for j in jobs]
        out = {}
        for jid, sid in ids:
            scores, statuses, _ = self.server.wait(sid, timeout_ms=600000)
            out[jid] = [float(s) for s in scores]
        return out

    def close(self):
        self.server.close()
