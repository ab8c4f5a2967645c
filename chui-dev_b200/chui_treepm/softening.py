"""Resolution of the reference's per-particle softening view into the
resolved epsilon lanes the C-ABI takes (chui_treepm_sources.softening and
chui_treepm_accumulator.target_softening).

The rules are those of include/cosmosim/gravity/tree_softening.hpp:
- a source takes its own epsilon where its override mask is set, else its
  species' epsilon when a species policy is enabled and species tags are
  given, else the configured epsilon (resolveSourceSofteningEpsilon,
  :152-180);
- the lane is materialized only when an epsilon lane, an override mask, or an
  enabled species policy with tags is present; otherwise every source takes
  the configured epsilon (sourceSofteningIsProvablyUniform,
  src/gravity/tree_gravity.cpp:82-94);
- a target takes its own epsilon where its override mask is set, else its
  species' epsilon (target tags), else -- with no target epsilon lane -- its
  source row's resolved epsilon, else its source row's species epsilon, else
  the configured one (targetSofteningEpsilonUnchecked, :90-110).
Values must be finite and non-negative (validatedSofteningEpsilon).
"""
from __future__ import annotations

import numpy as np

INVALID_ROW = 0xFFFFFFFF


def _check(values, what):
    v = np.asarray(values, dtype=np.float64)
    if not (np.isfinite(v).all() and (v >= 0.0).all()):
        raise ValueError(f"{what} must be finite and non-negative")
    return v


def resolve_sources(n: int, fallback: float, epsilon=None, override_mask=None, species_tag=None,
                    species_epsilon=None, species_enabled: bool = False):
    """Per-source epsilons (n doubles), or None when the sources are provably
    uniform (every source takes `fallback`)."""
    _check([fallback], "configured softening")
    has_eps = epsilon is not None and len(epsilon) > 0
    has_mask = override_mask is not None and len(override_mask) > 0
    has_species = species_enabled and species_tag is not None and len(species_tag) > 0
    if not (has_eps or has_mask or has_species):
        return None
    out = np.full(n, float(fallback))
    if has_species:
        tags = np.asarray(species_tag, dtype=np.int64)
        table = _check(species_epsilon, "species softening")
        if len(tags) != n or tags.min() < 0 or tags.max() >= len(table):
            raise ValueError("source species tags are outside the species table")
        out = table[tags].astype(np.float64)
    if has_eps and has_mask:
        eps = np.asarray(epsilon, dtype=np.float64)
        mask = np.asarray(override_mask) != 0
        if len(eps) != n or len(mask) != n:
            raise ValueError("source softening sidecars must match the source count")
        out = np.where(mask, _check(np.where(mask, eps, 0.0), "source softening override"), out)
    return out


def resolve_targets(rows, source_eps, n_sources: int, fallback: float, epsilon=None, override_mask=None,
                    species_tag=None, source_species_tag=None, species_epsilon=None,
                    species_enabled: bool = False):
    """Per-active-slot target epsilons, or None when the solver's own default
    (a target that is a source takes its source epsilon, others `fallback`)
    gives the same values. rows: the active slots' source rows
    (INVALID_ROW for independent targets); source_eps: resolve_sources()."""
    rows = np.asarray(rows, dtype=np.int64)
    has_eps = epsilon is not None and len(epsilon) > 0
    has_tspecies = species_enabled and species_tag is not None and len(species_tag) > 0
    has_sspecies = species_enabled and source_species_tag is not None and len(source_species_tag) > 0
    if not has_eps and not has_tspecies:
        # rule 3 (source row) and the fallback are the solver's default; only
        # species tags of rows outside the source lane would differ
        return None
    table = _check(species_epsilon, "species softening") if species_enabled else None
    out = np.full(len(rows), float(fallback))
    is_source = (rows >= 0) & (rows < n_sources)
    if not has_eps:
        src = source_eps if source_eps is not None else np.full(n_sources, float(fallback))
        out[is_source] = src[rows[is_source]]
    elif has_sspecies:
        tags = np.asarray(source_species_tag, dtype=np.int64)
        ok = is_source & (rows < len(tags))
        out[ok] = table[tags[rows[ok]]]
    if has_tspecies:
        out = table[np.asarray(species_tag, dtype=np.int64)].astype(np.float64)
    if has_eps and override_mask is not None and len(override_mask) > 0:
        eps = np.asarray(epsilon, dtype=np.float64)
        mask = np.asarray(override_mask) != 0
        out = np.where(mask, _check(np.where(mask, eps, 0.0), "target softening override"), out)
    return out
