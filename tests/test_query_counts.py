"""The opening query counts of every code level, restated in Python from
the reference's f64 formulas and compared with the host's at every chunk
size up to 30, in both fields.

The count of a level is min(ceil(-security / log2(1 - delta / 3)), rows)
(brakefold.rs:4-20), or all rows when no distance meets the security.  delta
is the QA distance bound (qafold.rs:79-178): the largest distance whose
failure bound is at most 2^-security, found by a 4096-step scan and 96
bisection steps and then shrunk by 1e-12, with log2 of the extension
field's size as the modulus.  The random-foldable layers are zero, so delta
is used as it is."""
import math

import pytest

import oracle
from test_oracle_claims import FIELDS

LN_2 = math.log(2.0)


def log_one_minus_exp(x):
    if x >= 0.0:
        return None
    return math.log1p(-math.exp(x)) if x < -LN_2 else math.log(-math.expm1(x))


def log_add_exp(a, b):
    m = max(a, b)
    return m + math.log(math.exp(a - m) + math.exp(b - m))


def qa_epsilon_at(m, index, d, ln_p):
    if m == 0 or index <= 1 or not (0.0 < d < 1.0) or not ln_p > 0.0:
        return None
    ln_p_minus_one = ln_p + math.log1p(-math.exp(-ln_p))
    g = 1.0 - d * ln_p_minus_one / ln_p + d * math.log(d) / ln_p + (1.0 - d) * math.log(1.0 - d) / ln_p
    eps = g - (1.0 + math.log(float(m)) / ln_p) / float(index)
    return eps if eps > 0.0 else None


def qa_bound_at(m, index, d, ln_p):
    eps = qa_epsilon_at(m, index, d, ln_p)
    if eps is None:
        return None
    ln_p_minus_one = ln_p + math.log1p(-math.exp(-ln_p))
    den = log_one_minus_exp(-float(index) * eps * ln_p)
    if den is None:
        return None
    den += ln_p_minus_one
    first_collision = float(index) * float(index - 1) * float(m) / 2.0
    first_collision_log = math.log(first_collision) - 2.0 * ln_p
    first_exponent = math.ceil(float(index - 1) / (float(index) * d)) * float(index) * eps
    first = log_add_exp(first_collision_log, -first_exponent * ln_p - den)
    second_collision_log = math.log(float(index) * float(m)) - ln_p
    second_exponent = math.ceil(1.0 / d) * float(index) * eps
    second = log_add_exp(second_collision_log, -second_exponent * ln_p - den)
    return eps, min(first, second)


def qa_distance_bound(m, index, security, modulus_log2):
    """The relative distance, or None when none meets the security."""
    ln_p = modulus_log2 * LN_2
    upper = 1.0 - 1.0 / float(index)
    target = -float(security) * LN_2

    def valid(d):
        r = qa_bound_at(m, index, d, ln_p)
        return r is not None and r[1] <= target

    lower, bracket = 0.0, upper
    for step in range(1, 4097):
        cand = upper * float(step) / 4096.0
        if valid(cand):
            lower = cand
        elif cand > lower:
            bracket = cand
            break
    if lower == 0.0:
        return None
    for _ in range(96):
        mid = (lower + bracket) * 0.5
        if valid(mid):
            lower = mid
        else:
            bracket = mid
    return lower * (1.0 - 1e-12)


def queries(security, d):
    return math.ceil(-float(security) / math.log2(1.0 - d / 3.0))


@pytest.mark.parametrize("field", ["f65521", "koalabear"])
def test_query_counts_match_the_restatement(field):
    p, deg = FIELDS[field][0], FIELDS[field][1]
    security = 100
    for chunk in (10, 12, 16, 20, 24, 26, 28, 30):
        rows, card_log2 = oracle.query_counts(chunk, 32, security, field=field)
        assert card_log2 == math.log2(float(p ** deg))
        for m, index, n, capped, unlimited in rows:
            assert index == 2 and n == m * index
            d = qa_distance_bound(m, index, security, card_log2)
            want = n if d is None else min(queries(security, d), n)
            assert capped == want, (chunk, m)
            assert unlimited == (2 ** 64 - 1 if d is None else queries(security, d)), (chunk, m)
