"""Owner -> GPU placement for serving on several GPUs, one process per GPU.

Each key owner's keys are registered on exactly one GPU and its requests run there, so no key
crosses NVLink and the data path needs no collective: the ranks serve disjoint owner sets.
The placement is a deterministic greedy balance of registered key bytes (largest owner first
onto the least-loaded rank, ties to the lower rank), so every rank computes the same table from
the same inputs without an exchange. The reference serves from one device and has no
counterpart; this is the multi-GPU form of its single-device server.
"""


class OwnerRouter:
    """rank_of[owner] for owners 0..len(key_bytes)-1 over `world` ranks."""

    def __init__(self, key_bytes, world):
        if world < 1:
            raise ValueError("world must be >= 1")
        if any(b < 0 for b in key_bytes):
            raise ValueError("key bytes must be >= 0")
        self.world = world
        self.rank_of = [0] * len(key_bytes)
        self.load = [0] * world
        for o in sorted(range(len(key_bytes)), key=lambda o: (-key_bytes[o], o)):
            r = min(range(world), key=lambda r: (self.load[r], r))
            self.rank_of[o] = r
            self.load[r] += key_bytes[o]

    def route(self, owner):
        return self.rank_of[owner]

    def owners_of(self, rank):
        """The owners placed on `rank`, in owner order."""
        return [o for o, r in enumerate(self.rank_of) if r == rank]

    def split(self, items, rank, owner_of):
        """The items (e.g. requests) whose owner is placed on `rank`, in their order."""
        return [it for it in items if self.rank_of[owner_of(it)] == rank]
