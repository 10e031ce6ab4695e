"""Text decks in front of the GPU run (the ``outdoor.*`` part of the
reference's ``load_text_input``, ``model/io/text_input.py:308-1035``).

A deck is ``key = value`` lines; ``#`` or ``;`` start a comment line, ``#``
also ends a value.  Keys are case-insensitive (stored lower-case).  Values
parse as the reference parses them: ``true/1/yes/y`` and ``false/0/no/n`` are
booleans (so ``= 1`` is ``True``), ``none/null/nan`` or empty are ``None``,
numbers are floats, anything else a string.

``case_from_deck`` merges a deck with keyword arguments with the driver's two
precedence rules (``spread_3d.py:972-1100``): for most keys a keyword given
explicitly wins over the deck (``_pick``), for the keys in ``DECK_FIRST`` the
deck wins over the keyword (``_deck_first``).
"""
from __future__ import annotations

from pathlib import Path

# spread_3d.py:1040-1100 _deck_first keys (deck value wins over the keyword)
DECK_FIRST = frozenset(k.lower() for k in (
    "dy", "n_z_bed", "turbulence_model", "combustion_closure", "chemistry_family",
    "boundary_condition_kind", "projection_method", "radiation_solver", "dom_subcycle_every",
    "lagrangian_bed_enable", "lagrangian_bed_N_per_cell", "lagrangian_bed_drying_mode",
    "lagrangian_bed_h_conv", "ignition_T_pin_enable", "ignition_T_pin_K",
    "ignition_T_pin_height_m", "ignition_T_pin_ramp_s", "ignition_T_pin_in_bed",
    "ignition_q_mult", "ignition_width_mult", "solid_phase_ignition_enable",
    "solid_phase_ignition_T_s_K", "level_set_passive", "edc_extinction_enable",
    "finney_tendril_enable", "nu_t_multiplier", "empirical_ros_enable", "empirical_ros_model",
    "empirical_ros_a_ch", "empirical_ros_u_threshold_m_s", "empirical_ros_blend_width_m_s",
    "empirical_ros_age_yr", "char_ox_flux_cap_W_m2", "char_ox_ash_exp", "moisture_jump_enable",
    "moisture_jump_t_s", "moisture_jump_delta_frac", "moisture_jump_x_lo_m",
    "moisture_jump_x_hi_m", "moisture_jump_z_lo_m", "moisture_jump_z_hi_m", "min_dt_s",
    "max_wall_time_s"))


def _parse_bool(text):
    v = text.strip().lower()
    if v in ("true", "1", "yes", "y"):
        return True
    if v in ("false", "0", "no", "n"):
        return False
    return None


def parse_value(text: str):
    """One deck value, typed as the reference's parser types it."""
    b = _parse_bool(text)
    if b is not None:
        return b
    v = text.strip()
    if v.lower() in ("none", "null", "nan", ""):
        return None
    try:
        return float(v)
    except ValueError:
        return v


def read_deck(path) -> dict:
    """``{"t_end": ..., "outdoor": {key: value}}`` from a deck file."""
    out = {"t_end": None, "outdoor": {}}
    for raw in Path(path).read_text(encoding="utf-8").splitlines():
        line = raw.strip()
        if not line or line.startswith("#") or line.startswith(";") or "=" not in line:
            continue
        key, value = (s.strip() for s in line.split("=", 1))
        if "#" in value:
            value = value[:value.index("#")].strip()
        kl = key.lower()
        if "sigma" in kl:
            continue
        if kl in ("t_end", "sim.t_end"):
            try:
                out["t_end"] = float(value)
            except ValueError:
                out["t_end"] = None
        elif kl.startswith("outdoor."):
            out["outdoor"][kl.split(".", 1)[1]] = parse_value(value)
    return out


def case_from_deck(path, wind_speed_m_s: float = 0.0, **kwargs) -> dict:
    """A case dict (deck keys + ``wind_speed_m_s``) for ``run_3d_spread_gpu``
    from a deck file and keyword overrides.  ``None`` keywords are ignored,
    as the driver ignores unset keywords."""
    deck = read_deck(path)["outdoor"]
    case = {k: v for k, v in deck.items() if v is not None}
    for k, v in kwargs.items():
        if v is None:
            continue
        kl = k.lower()
        if kl in DECK_FIRST and kl in case:
            continue
        case.pop(kl, None)
        case[k] = v
    case["wind_speed_m_s"] = float(wind_speed_m_s)
    return case
