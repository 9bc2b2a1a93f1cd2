"""Plain-text Pearl input files for the command-line tests.

The physical values are those of the reference's example inputs
(examples/fe_c_phase_diagram_10K.in, fe_c_eutectoid.in,
legacy_direct/fe_c_137.in); grids and times are shrunk so that runs take
seconds.  Each case is a list of (key, value) lines in input-file order.
"""
from __future__ import annotations

from pathlib import Path

COMMON = [
    ("Vm", "1e-6"), ("epsilon", "14e-9"), ("sigma", "0.5"), ("triple", "10"),
    ("tau_at", "1.72402799784e8"), ("tau_ag", "1.72402799784e8"), ("tau_tg", "7.11828875478e9"),
]

PHASE_DIAGRAM_10K = [
    ("thermo_mode", "eutectoid_reference"), ("T_eutectoid", "999.68459774"), ("undercooling", "10"),
    ("temperature_law", "phase_diagram_fixed_curvature"), ("max_undercooling", "10"),
    ("Aeq_alpha", "4724862.6373624019"), ("Beq_alpha", "22964.296428571855"), ("Ceq_alpha", "-42255.03701292308"),
    ("D_alpha", "2e-9"),
    ("Aeq_theta", "100000000"), ("Beq_theta", "-49968654.66102279"), ("Ceq_theta", "6207741.2462954065"),
    ("D_theta", "2e-9"),
    ("Aeq_gamma", "172591.65731409981"), ("Beq_gamma", "19450.725112218221"), ("Ceq_gamma", "-42053.816371518253"),
    ("D_gamma", "1e-9"),
    ("ceq_alpha", "0.00088690859310575857"), ("ceq_theta", "0.25"), ("ceq_gamma", "0.034458832049305582"),
    ("slope_alpha_on_alpha_gamma", "-4.6282639461434345e-06"),
    ("slope_gamma_on_alpha_gamma", "-0.00031198492411304955"),
    ("slope_theta_on_theta_gamma", "0"), ("slope_gamma_on_theta_gamma", "0.00010753713136114516"),
]

LINEAR_GP = [
    ("thermo_mode", "eutectoid_reference"), ("T_eutectoid", "999.76"), ("undercooling", "10.0"),
    ("temperature_law", "linear_gp"), ("max_undercooling", "10.0"),
    ("Aeq_alpha", "2.110387326850582194E+5"), ("Beq_alpha", "4.035447487350817940E+3"),
    ("Ceq_alpha", "-5.946151226167807263E+3"), ("dq2_dT_alpha", "-7.897444442197080000E-8"),
    ("dq1_dT_alpha", "6.895916700000000000E-4"), ("dq0_dT_alpha", "-1.089458632862000000E+1"), ("D_alpha", "2e-9"),
    ("Aeq_theta", "1.315789473684210526E+7"), ("Beq_theta", "-6.574538381578947368E+6"),
    ("Ceq_theta", "8.164221038271662664E+5"), ("dq2_dT_theta", "0.0"), ("dq1_dT_theta", "2.146300000000000000E-7"),
    ("dq0_dT_theta", "-8.688560674440000000E+0"), ("D_theta", "2e-9"),
    ("Aeq_gamma", "2.462118547480502910E+4"), ("Beq_gamma", "2.713423471716552040E+3"),
    ("Ceq_gamma", "-5.917127514474751428E+3"), ("dq2_dT_gamma", "-2.111000000000000000E-17"),
    ("dq1_dT_gamma", "9.357150000000000000E-6"), ("dq0_dT_gamma", "-9.949361760240000000E+0"), ("D_gamma", "1e-9"),
]

DIRECT = [
    ("thermo_mode", "direct_at_temperature"), ("temperature", "989.76"),
    ("A_alpha", "6.331161979528086e5"), ("B_alpha", "3.374509335088470e3"), ("C_alpha", "-5.852000117829494e3"),
    ("D_alpha", "2e-9"),
    ("A_theta", "1.315789473684211e7"), ("B_theta", "-6.574594863157894e6"), ("C_theta", "8.165231004262522e5"),
    ("D_theta", "2e-9"),
    ("A_gamma", "2.462118547531691e4"), ("B_gamma", "2.708815789259557e3"), ("C_gamma", "-5.817887580401304e3"),
    ("D_gamma", "1e-9"),
]


def grid(nx: int, ny: int, dx: str = "2.79e-9", dt: str = "4e-12", end: str = "1e-9", out: str = "2e-10"):
    return [("nx", str(nx)), ("ny", str(ny)), ("dx", dx), ("dt", dt), ("dt_max", dt), ("dt_min", "1e-16"),
            ("end_time", end), ("output_dt", out)]


def case_sharp_smooth():
    return PHASE_DIAGRAM_10K + grid(64, 48) + COMMON + [
        ("initialization", "sharp_smooth"), ("seed_height", "33e-9"), ("theta_columns", "9"),
        ("gamma_carbon", "0.034458832049305582"), ("smooth_steps", "30"), ("smooth_min_steps", "30")]


def case_lamella_linear_gp():
    return LINEAR_GP + grid(48, 64) + COMMON + [
        ("initialization", "lamella"), ("seed_height", "40e-9"), ("theta_columns", "7"), ("gamma_carbon", "0.034433")]


def case_direct_flat_mean():
    return DIRECT + grid(40, 40) + COMMON + [
        ("initialization", "flat"), ("seed_height", "30e-9"), ("phase_a", "0"), ("phase_b", "2"),
        ("mean_carbon", "0.03")]


def case_microsim():
    return PHASE_DIAGRAM_10K + grid(64, 40) + COMMON + [
        ("initialization", "microsim"), ("FILLCUBE", "{1,0,0,0,7,9,0};"), ("FILLCUBE", "{0,8,0,0,63,9,0};"),
        ("gamma_carbon", "0.034458832049305582"), ("smooth_steps", "20"), ("smooth_min_steps", "20")]


def case_moving_window():
    return PHASE_DIAGRAM_10K + grid(48, 40, end="6e-10", out="1e-10") + COMMON + [
        ("initialization", "lamella"), ("seed_height", "64e-9"), ("theta_columns", "7"),
        ("gamma_carbon", "0.034458832049305582"), ("moving_window", "1"), ("shift_trigger", "60e-9"),
        ("shift_target", "40e-9")]


def case_smoke():
    """The key-values of the reference's start-up check examples/fe_c_phase_diagram_10K_smoke.in
    (137x250, sharp_smooth, to 0.015 microseconds: ~5,500 adaptive steps)."""
    return PHASE_DIAGRAM_10K + grid(137, 250, dt="1.5e-11", end="1.5e-8", out="2.5e-8") + COMMON + [
        ("initialization", "sharp_smooth"), ("seed_height", "58.59e-9"), ("theta_columns", "17"),
        ("gamma_carbon", "0.034458832049305582"), ("smooth_steps", "100"), ("smooth_min_steps", "100"),
        ("smooth_energy_rtol", "1e-10"), ("smooth_max_phase_change", "0.02")]


# Filling commands of every method, on the 137x250 grid of the reference's
# examples (values chosen off the grid lines, angles off the axes, so that the
# cells near the painted boundaries test the arithmetic).
FILL_CASES = {
    # the reference's G137 sharp geometry: 17 theta and 120 alpha columns in rows 0..20
    "cube_g137": [("FILLCUBE", "{1,0,0,0,16,20,0};"), ("FILLCUBE", "{0,17,0,0,136,20,0};")],
    "cylinders": [("FILLCYLINDER", "{0,68,125,0,0,40.5}"), ("FILLCYLINDER", "{1,68,125,0,0,13.7}"),
                  ("FILLCYLINDER", "{0,20,200,0,0,9}")],
    "center_box": [("FILLCENTERBOX2D", "{10,127,30,220,1,0}"), ("FILLCUBE", "{2,0,0,0,5,5,0}"),
                   ("FILLCUBE", "{1,60,100,0,70,140,0}")],
    "y_junction": [("FILLYJUNCTION2D", "{0,137,0,250,68,125,90,210,330,120,14.5,0,2}")],
    "y_junction_lamellae": [("FILLYJUNCTIONLAMELLAE2D", "{5,130,10,240,70,120,17,137,257,110,20,7.3,1.9,0,1,2}")],
    "adhered_arm": [("FILLADHEREDPEARLITEARM2D", "{12.5,30,63.4,160,9,0.125,6.5,2.25,4,0,1}")],
    "adhered_arm_steep": [("FILLADHEREDPEARLITEARM2D", "{120.25,10.5,121.7,180,14,0.2,5.5,0,0,1,0}")],
    "ellipse": [("FILLPEARLITEELLIPSE2D", "{68.5,20.25,77,10,12,14.2,0.35,0.13,5,0,1}")],
    "ellipse_rotated": [("FILLPEARLITEELLIPSE2D", "{30,200,-33.3,0,7,11.1,0.6,0.3,0,1,0}")],
    "sequence": [("FILLCENTERBOX2D", "{0,137,0,250,0,2}"),
                 ("FILLYJUNCTION2D", "{20,120,40,200,70,120,45,165,285,90,8.5,1,2}"),
                 ("FILLCYLINDER", "{0,70,120,0,0,6.25}"),
                 ("FILLADHEREDPEARLITEARM2D", "{70,120,-90,100,5,0.3,4,1.5,3.5,1,0}"),
                 ("FILLPEARLITEELLIPSE2D", "{100,60,15,2,5,9.7,0.5,0.2,2,0,1}"),
                 ("FILLCUBE", "{1,130,240,0,136,249,0}")],
}


def case_fill(name: str):
    """A microsim input painting FILL_CASES[name] on 137x250 (one smoothing step)."""
    return PHASE_DIAGRAM_10K + grid(137, 250) + COMMON + [
        ("initialization", "microsim"), *FILL_CASES[name], ("gamma_carbon", "0.034458832049305582"),
        ("smooth_steps", "1"), ("smooth_min_steps", "1")]


def fill_params(value: str) -> list[float]:
    """The numbers of a filling command's value "{a,b,...};"."""
    v = value.strip().rstrip(";").strip()
    assert v[0] == "{" and v[-1] == "}"
    return [float(t) for t in v[1:-1].split(",")]


VALID = {
    "sharp_smooth": case_sharp_smooth,
    "lamella_linear_gp": case_lamella_linear_gp,
    "direct_flat_mean": case_direct_flat_mean,
    "microsim": case_microsim,
    "moving_window": case_moving_window,
}


def _edit(lines, drop=(), set_=None, add=()):
    out = [(k, v) for k, v in lines if k not in drop]
    if set_:
        out = [(k, set_.get(k, v)) for k, v in out]
    return out + list(add)


def invalid_cases() -> dict[str, list]:
    base = case_sharp_smooth()
    fill = [("FILLCUBE", "{1,0,0,0,7,9,0};")]
    micro = _edit(base, set_={"initialization": "microsim"})
    return {
        "missing_key": _edit(base, drop=("sigma",)),
        "duplicate_key": base + [("sigma", "0.5")],
        "unknown_key": base + [("colour", "blue")],
        "bad_number": _edit(base, set_={"dx": "2.79e-9x"}),
        "unparsable_number": _edit(base, set_={"dx": "abc"}),
        "bad_integer": _edit(base, set_={"nx": "64.5"}),
        "no_mode": _edit(base, drop=("thermo_mode",)),
        "bad_law": _edit(base, set_={"temperature_law": "cubic"}),
        "undercooling_out_of_range": _edit(base, set_={"undercooling": "11"}),
        "two_compositions": base + [("initial_mu", "3e4")],
        "bad_mode": base + [("mode", "thermal")],
        "unknown_initialization": _edit(base, set_={"initialization": "spiral"}),
        "fill_without_microsim": base + fill,
        "microsim_without_fill": micro,
        "fill_bad_bounds": micro + [("FILLCUBE", "{1,0,0,0,80,9,0};")],
        "fill_bad_phase": micro + [("FILLCUBE", "{3,0,0,0,7,9,0};")],
        "fill_malformed": micro + [("FILLCUBE", "{1,0,,0,7,9,0}")],
        "fill_unsupported": micro + [("FILLSPHERE", "{1,2,3}")],
        "fill_multigrain": micro + [("FILLTHREEGRAINYJUNCTION2D", "{1,2,3}")],
        "fill_cylinder_z": micro + [("FILLCYLINDER", "{0,10,10,1,0,4}")],
        "fill_box_phases": micro + [("FILLCENTERBOX2D", "{0,10,0,10,1,1}")],
        "fill_yjunction_count": micro + [("FILLYJUNCTION2D", "{0,10,0,10,5,5,0,120,240,4,2}")],
        "fill_arm_fraction": micro + [("FILLADHEREDPEARLITEARM2D", "{10,10,0,20,4,1.5,2,1,0,0,1}")],
        "fill_ellipse_phases": micro + [("FILLPEARLITEELLIPSE2D", "{10,10,0,0,3,8,0.5,0.2,0,1,1}")],
        "bad_seed": _edit(base, set_={"theta_columns": "64"}),
        "bad_time": _edit(base, set_={"dt_max": "1e-12"}),
        "bad_control": base + [("max_phase_change", "0.5")],
        "bad_smoothing": _edit(base, set_={"smooth_min_steps": "31"}),
        "bad_window": base + [("moving_window", "1"), ("shift_trigger", "10e-9"), ("shift_target", "20e-9")],
        "bad_phase_pair": base + [("phase_a", "2")],
        "bad_interface": _edit(base, set_={"sigma": "-0.5"}),
        "bad_tau": _edit(base, set_={"tau_tg": "0"}),
        "missing_equals": base + [("just text", None)],
        "direct_bad_parabola": _edit(case_direct_flat_mean(), set_={"A_theta": "-1"}),
        "direct_bad_temperature": _edit(case_direct_flat_mean(), set_={"temperature": "0"}),
    }


def write_input(path: Path, lines) -> Path:
    text = []
    for k, v in lines:
        text.append(k if v is None else f"{k} = {v}")
    path.write_text("# generated test input\n" + "\n".join(text) + "\n")
    return path
