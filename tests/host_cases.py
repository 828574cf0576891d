"""Case directories in the reference's file layout (mesh/structuredMesh.info,
case/case.info, case/initialConditions.info) for the C++ host-layer tests, written from a
CaseSpec so that the host layer's parse can be compared with the Python case record."""
from __future__ import annotations

import os

from caffe_old_b200 import cases as C


def _vec(v):
    return "(" + ",".join(repr(float(x)) for x in v) + ")"


def write_case(root: str, spec: C.CaseSpec, lengths, nodes_ijk, steps: int, write_interval: int = 1000, extra: str = "",
               run_control_extra: str = "", initial_conditions: str | None = None) -> None:
    os.makedirs(os.path.join(root, "mesh"), exist_ok=True)
    os.makedirs(os.path.join(root, "case"), exist_ok=True)
    lx, ly, lz = lengths
    verts = [(0, 0, 0), (lx, 0, 0), (lx, ly, 0), (0, ly, 0), (0, 0, lz), (lx, 0, lz), (lx, ly, lz), (0, ly, lz)]
    with open(os.path.join(root, "mesh", "structuredMesh.info"), "w") as f:
        f.write("; generated case\nMeshName testMesh\nMetricConversion 1.\n\nVertices\n{\n")
        for q, v in enumerate(verts):
            f.write(f"\tv{q + 1} {_vec(v)}\n")
        f.write("}\n\nResolution " + "(" + ",".join(str(n) for n in nodes_ijk) + ")\n")
    with open(os.path.join(root, "case", "case.info"), "w") as f:
        f.write("; generated case\n\nRunControl\n{\n\tterminationCondition iterations\n"
                f"\tmaxNumberOfIterations {steps + 1}\n\tfileWriteInterval {write_interval}\n\ttimeStep {spec.dt!r}\n"
                "\tmaxSimTime 48\n\tmaxRealTimeHours 48\n" + run_control_extra + "}\n\n")
        f.write("Solver\n{\n\ttimeAccurate " + ("ON" if spec.time_accurate else "OFF") + "\n"
                f"\trelaxationFactorMomentum {spec.omega_u!r}\n\trelaxationFactorPCorr {spec.omega_p!r}\n"
                f"\trho {spec.rho!r}\n\tmu {spec.mu!r}\n\tnumberOfPressureCorrections {spec.n_pcorr}\n"
                f"\tnumberOfInnerIterations {spec.n_inner}\n\tconvectionScheme {spec.convection}\n"
                "\tnonOrthogonalCorrection " + ("ON" if spec.nonorth else "OFF") + "\n}\n\n")
        f.write("LinearSolvers\n{\n"
                f"\tmomentum {spec.mom_method}\n\tpressureCorrection {spec.p_method}\n\ttolerance {spec.p_rtol!r}\n"
                f"\tmaxIterations {spec.maxit}\n\tpressureCorrectionForm {spec.p_form}\n}}\n\n")
        if spec.kind == "ibpiso":
            f.write("ImmersedBoundaries\n{\n\tSphere\n\t{\n"
                    f"\t\tradius {spec.ib_radius!r}\n\t\tcenter {_vec(spec.ib_center)}\n\t}}\n}}\n\n")
        f.write("Boundaries\n{\n")
        for face, typ, rv, rval in zip(C.FACES, spec.bc, spec.ref_vec, spec.ref_val):
            f.write(f"\t{face}\n\t{{\n\t\ttype {typ}\n\t\trefVector {_vec(rv)}\n\t\trefValue {float(rval)!r}\n\t}}\n")
        f.write("}\n" + extra)
    with open(os.path.join(root, "case", "initialConditions.info"), "w") as f:
        if initial_conditions is not None:
            f.write(initial_conditions)
        else:
            f.write(f"u\n{{\n\ttype uniform\n\tvalue {_vec(spec.u_init)}\n}}\n\np\n{{\n\ttype uniform\n\tvalue {float(spec.p_init)!r}\n}}\n")


def read_tec360_fields(path: str, n_cells: int) -> dict:
    """Cell fields of the last zone of a solution file written by HexaFvmMesh::writeTec360, by the
    names of its VARIABLES line ("p", "massFlow", "u_x", ...)."""
    import re
    with open(path) as f:
        text = f.read()
    names = re.findall(r'"([^"]+)"', text.split("\n", 2)[1])
    last = text.split("ZONE")[-1]
    header, body = last.split("\n", 1)
    vals = [float(x) for x in body.split()]
    ni, nj, nk = (int(re.search(rf"{a} = (\d+)", header).group(1)) for a in "IJK")
    off = 3 * ni * nj * nk
    out = {}
    for q, nm in enumerate(names[3:]):
        out[nm] = vals[off + q * n_cells:off + (q + 1) * n_cells]
    return out


def read_tec360_last_zone(path: str, n_cells: int):
    """(p, u planes) of the last zone of a solution file written by HexaFvmMesh::writeTec360."""
    f = read_tec360_fields(path, n_cells)
    return f["p"], f["u_x"] + f["u_y"] + f["u_z"]
