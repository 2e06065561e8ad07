import time
perf_counter = time.perf_counter
process_clock = time.process_time
QUIET, ERROR, WARN, NOTE, INFO, DEBUG, DEBUG1, DEBUG2, DEBUG3, DEBUG4 = 0, 1, 2, 3, 4, 5, 6, 7, 8, 9


class Logger:
    def __init__(self, stdout=None, verbose=0):
        self.verbose = verbose

    def _p(self, *a, **k):
        pass
    error = warn = note = info = debug = debug1 = debug2 = debug3 = debug4 = _p


def new_logger(obj=None, verbose=0):
    return Logger(verbose=verbose)


def timer_debug1(obj, msg, *t0):
    return (process_clock(), perf_counter())


def _noop(*a, **k):
    pass


debug = debug1 = note = info = warn = error = _noop
