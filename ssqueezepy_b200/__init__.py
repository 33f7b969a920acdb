# -*- coding: utf-8 -*-
"""B200-native synchrosqueezing hot path (ssq_cwt / cwt / ssq_stft / stft /
icwt) with ssqueezepy's signatures and return tuples."""
