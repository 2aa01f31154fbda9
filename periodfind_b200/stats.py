"""Result containers: Statistics and Periodogram.

Behaviour follows the reference's periodfind/__init__.py:253-546: the best
`n` trial parameters by np.argpartition (minimum for CE, maximum for AOV and
LS), periodogram-wide mean / std / median / MAD, and a significance computed
as |value - mean| / std ('stdmean') or |value - median| / mad ('madmedian').
"""

import numpy as np


class Statistics:
    """Statistics of one trial-parameter set within a periodogram."""

    def __init__(self, params, value, mean, std, median, mad, significance_type="stdmean"):
        self.params = params
        self.value = value
        self.mean = mean
        self.std = std
        self.median = median
        self.mad = mad
        self.significance_type = significance_type

    def __repr__(self):
        return (
            f"Statistics(params={self.params}, value={self.value:.6g}, "
            f"significance_type='{self.significance_type}')"
        )

    @property
    def significance(self):
        if self.significance_type == "stdmean":
            return abs(self.value - self.mean) / self.std
        if self.significance_type == "madmedian":
            return abs(self.value - self.median) / self.mad
        raise NotImplementedError("Statistic " + self.significance_type + " not implemented")

    @staticmethod
    def statistics_from_data(data, params, use_max, mean=None, std=None, median=None,
                             mad=None, n=1, significance_type="stdmean"):
        """Statistics for the best `n` entries of periodogram `data`.

        Returns one Statistics when n == 1, else a list sorted best-first.
        """
        if not use_max:
            part = np.argpartition(data, n, axis=None)[:n]
        else:
            part = np.argpartition(data, len(data) - n, axis=None)[-n:]
        idxs = np.unravel_index(part, data.shape)
        values = data[idxs]
        if mean is None:
            mean = np.mean(data)
        if std is None:
            std = np.std(data)
        if median is None:
            median = np.median(data)
        if mad is None:
            mad = np.median(np.abs(data - median))
        best = []
        for k in range(n):
            idx = tuple(dim[k] for dim in idxs)
            param = [params[i][idx[i]] for i in range(len(params))]
            best.append(Statistics(param, values[k], mean, std, median, mad, significance_type))
        best.sort(key=lambda s: s.value, reverse=use_max)
        return best[0] if n == 1 else best


class Periodogram:
    """A full periodogram with its trial parameters."""

    def __init__(self, periodogram, params, use_max):
        self.use_max = use_max
        self.data = periodogram
        self.params = params
        self.mean = None
        self.std = None
        self.median = None
        self.mad = None

    def __repr__(self):
        shape = self.data.shape if hasattr(self.data, "shape") else "?"
        return f"Periodogram(shape={shape}, use_max={self.use_max})"

    def _calc_mean(self):
        if self.mean is None:
            self.mean = np.mean(self.data)

    def _calc_std(self):
        if self.std is None:
            self.std = np.std(self.data)

    def _calc_median(self):
        if self.median is None:
            self.median = np.median(self.data)

    def _calc_mad(self):
        if self.mad is None:
            self.mad = np.median(np.abs(self.data - self.median))

    def best_params(self, n=1, significance_type="stdmean"):
        """Statistics for the best `n` trial parameters of this periodogram."""
        self._calc_mean()
        self._calc_std()
        self._calc_median()
        self._calc_mad()
        return Statistics.statistics_from_data(
            self.data, self.params, self.use_max, mean=self.mean, std=self.std,
            median=self.median, mad=self.mad, n=n, significance_type=significance_type)
