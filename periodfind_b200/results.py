"""Result objects of periodfind_b200.gpu: Statistics and Periodogram.

They carry the interface periodfind's own classes have
(periodfind/__init__.py:253-546), because callers of the reference read
it: the constructor arguments and attribute names, `significance` by
'stdmean' (|value - mean| / std) or 'madmedian' (|value - median| / mad),
`Statistics.statistics_from_data`, `Periodogram.best_params`, and the same
picks and order of the best cells.  Inside the periodfind package the
drop-in modules (periodfind_b200/dropin) return the package's own classes
instead; these serve periodfind_b200.gpu used on its own.
"""

from __future__ import annotations

import operator

import numpy as np

# Significance of a value against its periodogram, by name.
_SIGNIFICANCE = {
    "stdmean": lambda s: abs(s.value - s.mean) / s.std,
    "madmedian": lambda s: abs(s.value - s.median) / s.mad,
}


def _summary(data, mean=None, std=None, median=None, mad=None):
    """(mean, std, median, mad) of a periodogram, numpy's values; the ones
    given are kept (mad is taken about the median, given or computed)."""
    mean = np.mean(data) if mean is None else mean
    std = np.std(data) if std is None else std
    median = np.median(data) if median is None else median
    mad = np.median(np.abs(data - median)) if mad is None else mad
    return mean, std, median, mad


def _picked_cells(data, use_max, n):
    """Flat indices of the n cells the reference reports, in its order
    before sorting: np.argpartition at n for a minimum; for a maximum, the
    last n of the partition at len(data) - n.  len() counts the first axis
    (trial periods), not the cells, so with several period derivatives the
    maximum side reports n cells of the upper part of the partition, which
    need not be the n largest; kept so that results stay the reference's."""
    if use_max:
        return np.argpartition(data, len(data) - n, axis=None)[-n:]
    return np.argpartition(data, n, axis=None)[:n]


class Statistics:
    """One trial-parameter set of a periodogram: its parameters, its value,
    and the periodogram's mean, std, median and median absolute deviation."""

    def __init__(self, params, value, mean, std, median, mad, significance_type="stdmean"):
        self.params = params
        self.value = value
        self.mean = mean
        self.std = std
        self.median = median
        self.mad = mad
        self.significance_type = significance_type

    def __repr__(self):
        return (f"Statistics(params={self.params}, value={self.value:.6g}, "
                f"significance_type='{self.significance_type}')")

    @property
    def significance(self):
        rule = _SIGNIFICANCE.get(self.significance_type)
        if rule is None:
            raise NotImplementedError("Statistic " + self.significance_type + " not implemented")
        return rule(self)

    @staticmethod
    def statistics_from_data(data, params, use_max, mean=None, std=None, median=None,
                             mad=None, n=1, significance_type="stdmean"):
        """Statistics of the best n cells of `data` (one Statistics for n ==
        1, else a list, best first); params[d] holds the trial values of
        axis d."""
        coords = np.unravel_index(_picked_cells(data, use_max, n), data.shape)
        values = data[coords]
        summary = _summary(data, mean, std, median, mad)
        found = [Statistics([params[d][coords[d][k]] for d in range(len(params))], values[k],
                            *summary, significance_type) for k in range(n)]
        found.sort(key=operator.attrgetter("value"), reverse=use_max)
        return found[0] if n == 1 else found


class Periodogram:
    """A whole periodogram with its trial parameters.  mean, std, median and
    mad stay None until best_params() first needs them."""

    def __init__(self, periodogram, params, use_max):
        self.use_max = use_max
        self.data = periodogram
        self.params = params
        self.mean = self.std = self.median = self.mad = None

    def __repr__(self):
        shape = getattr(self.data, "shape", "?")
        return f"Periodogram(shape={shape}, use_max={self.use_max})"

    def best_params(self, n=1, significance_type="stdmean"):
        """Statistics of the best n trial parameters (see
        Statistics.statistics_from_data)."""
        self.mean, self.std, self.median, self.mad = _summary(
            self.data, self.mean, self.std, self.median, self.mad)
        return Statistics.statistics_from_data(self.data, self.params, self.use_max,
                                               self.mean, self.std, self.median, self.mad, n,
                                               significance_type)
