"""``cupy.cuda`` stand-in with host-clock events (oracle test infrastructure)."""

import time as _time


class Event:
    def __init__(self, *args, **kwargs):
        self.t = None

    def record(self, stream=None):
        self.t = _time.perf_counter()

    def synchronize(self):
        return None


def get_elapsed_time(start, end):
    return (end.t - start.t) * 1e3


class _Runtime:
    @staticmethod
    def deviceSynchronize():
        return None


runtime = _Runtime()
