"""moldyn_run's thermo CSV from the library (apps/moldyn_run.cpp:229-245 header,
497-511 rows, 600-617 column header), on the CPU: the header lines and the rows
for given thermo values equal a restatement of StepSampler::record formatted as
the reference's stream (std::setprecision(10), default float format == %.10g),
with the tail corrections from the oracle (lennard_jones.cpp:121-151)."""
import numpy as np
import pytest

import moleculardynamics_b200 as md
import oracle as O


def g10(x):
    return "%.10g" % x


@pytest.mark.parametrize("trunc", [0, 1])
def test_thermo_csv_rows_restate_the_reference(tmp_path, trunc):
    n, box, dt = 864, np.array([10.0776, 10.0776, 10.0776]), 0.005
    rng = np.random.default_rng(3)
    rows = np.column_stack([rng.normal(-5000, 30, 7), rng.normal(1000, 50, 7),
                            rng.normal(900, 10, 7), rng.normal(0, 1, 7)])
    lj = md.LennardJones(1.0, 1.0, 2.5, trunc)
    path = tmp_path / "thermo.csv"
    csv = md.ThermoCsv(path, command_line="moldyn_run --cells 6", revision="abc123",
                       host="box", truncation=trunc, dof_langevin=3 * n, dof_nve=3 * n - 3)
    csv.append(lj, n, box, rows[:3], first_step=0, dt=dt, phase="equilibrate", dof=3 * n)
    csv.append(lj, n, box, rows[3:], first_step=100, dt=dt, phase="production", dof=3 * n - 3,
               step_stride=10)
    csv.close()
    lines = path.read_text().splitlines()
    tail = trunc == 0
    assert lines[:4] == ["# command: moldyn_run --cells 6", "# git_sha: abc123", "# host: box",
                         "# units: reduced Lennard-Jones units (sigma = epsilon = mass = kB = 1)"]
    assert lines[4] == "# truncation: " + ("truncated" if tail else "linear-force-shift")
    assert lines[5] == "# pressure_includes_tail_correction: " + ("yes" if tail else "no")
    assert lines[6] == "# potential_energy_includes_tail_correction: " + ("yes" if tail else "no")
    assert lines[7].startswith(f"# temperature_dof: 3N={3 * n} while Langevin drives")
    assert f"3N-3={3 * n - 3} under the momentum-conserving" in lines[7]
    assert lines[8] == "step,time,phase,potential_energy,kinetic_energy,total_energy,temperature,pressure"
    u_lrc, p_lrc = O.lj_lrc(n, box, rc=2.5, trunc=trunc)
    if not tail:
        u_lrc = p_lrc = 0.0
    volume = box[0] * box[1] * box[2]
    want = []
    for k, r in enumerate(rows):
        step, phase, dof = (k, "equilibrate", 3 * n) if k < 3 else (100 + 10 * (k - 3), "production", 3 * n - 3)
        t = step * dt
        temp = 2.0 * r[2] / dof
        pres = (n / volume) * temp + r[1] / (3.0 * volume) + p_lrc
        pe = r[0] + u_lrc
        want.append(",".join([str(step), g10(t), phase, g10(pe), g10(r[2]), g10(pe + r[2]),
                              g10(temp), g10(pres)]))
    assert lines[9:] == want


def test_thermo_csv_unwritable_path_is_a_runtime_error(tmp_path):
    with pytest.raises(md.MDError, match="cannot open"):
        md.ThermoCsv(tmp_path / "missing" / "thermo.csv")
