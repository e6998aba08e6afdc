"""Drive the compiled TENSUM reference (oracle/_ref) on a synthetic case.

Test infrastructure only (the oracle is the checker, never the product):
used to generate golden fixtures in a container that has the reference
sources, and by the reference arm of bench.py to time the reference's own CPU
code.  It writes a ``param.in`` in the reference's section format
(src/parameter.cc:16-33, readme/README.md "Description of param.in"), a
single-partition part file, an optional initial-condition file, runs
``oracle/_ref/tensum_harness`` and parses its dump.
"""
from __future__ import annotations

import os
import struct
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
HARNESS = os.path.join(HERE, "_ref", "tensum_harness")

RECON_NAMES = {"first", "second", "second_muscl", "minmod", "tvb_minmod", "eno2", "van_albada"}
FLUX_NAMES = {"kepes_tecno_roe", "kepes_tecno_rusanov", "kepec", "kep", "roe_ec", "simple_avg"}


def harness_available() -> bool:
    return os.access(HARNESS, os.X_OK)


def param_text(cfg: dict) -> str:
    """Render a param.in for the reference from a flat config dict.

    Keys: flux, reconstruct, tvb_M, model ('euler'|'ns'), mu_ref, prandtl,
    gamma, gas_const, cfl, time_mode, time_step, final_time, max_iter,
    time_stamps, ev_alpha, ev_beta, boundary: {tag: (type, {var: expr})}.
    Monte Carlo keys: samples (list of sample ids), rnd_per_sample,
    ic ({variable: fparser expression}), constants ({name: value}),
    online_stat (bool), variables (extra moment variables, e.g. ["density"]).
    forces: {name: [face tags]} (integrals section, compute_forces).
    liou_fix (bool), bc_scheme ('weak' | 'strong').
    Output keys: files (bool: solution, log, global and restart files),
    surfaces (face tags of the surface files).  cell: 'median' | 'voronoi' dual cells.
    axisymmetric (bool): the run uses the reference's -axi option (radius = x).
    """
    flux = cfg.get("flux", "kepes_tecno_roe")
    recon = cfg.get("reconstruct", "minmod")
    assert flux in FLUX_NAMES and recon in RECON_NAMES
    # second_muscl has no parameter-file keyword: the file names "second" and the
    # harness switches the scheme (TENSUM_HARNESS_RECON, set by run_case)
    rec = f"      method   {'second' if recon == 'second_muscl' else recon}\n"
    if recon == "tvb_minmod":
        rec += f"      M_value  {cfg.get('tvb_M', 1.0):.17g}\n"
    model = cfg.get("model", "euler")
    bnd = []
    for tag, (btype, vals) in sorted(cfg["boundary"].items()):
        body = "\n".join(f"      {k}   {v}" for k, v in vals.items())
        bnd.append(f"   {tag}\n   {{\n      type   {btype}\n{body}\n   }}")
    bnd_text = "\n".join(bnd)
    samples = "\n".join(f"         {int(s)}" for s in cfg.get("samples", []))
    ic = cfg.get("ic", {})
    ic_text = "\n".join(f"   {v}  {ic.get(v, d)}" for v, d in (("temperature", "1.0"), ("xvelocity", "0.0"),
                                                                ("yvelocity", "0.0"), ("zvelocity", "0.0"),
                                                                ("pressure", "1.0")))
    consts = cfg.get("constants", {"dummy": 0.0})
    const_text = "\n".join(f"   {k} {v:.17g}" for k, v in consts.items())
    var_text = "\n".join(f"      {v}" for v in cfg.get("variables", []))
    force_text = "\n".join("   force\n   {\n      " + name + "   " + "   ".join(str(t) for t in tags) + "\n   }"
                           for name, tags in cfg.get("forces", {}).items())
    online = "yes" if cfg.get("online_stat", False) else "no"
    files = "yes" if cfg.get("files", False) else "no"
    surf_text = "\n".join(f"      {int(t)}" for t in cfg.get("surfaces", []))
    return f"""grid
{{
   cell      {cfg.get('cell', 'median')}
}}

numeric
{{
   time_mode    {cfg.get('time_mode', 'unsteady')}
   time_scheme  {cfg.get('time_scheme', 'ssprk3')}
   time_step    {cfg.get('time_step', 0.0):.17g}
   cfl          {cfg.get('cfl', 0.8):.17g}
   max_iter     {cfg.get('max_iter', 1000000000)}
   final_time   {cfg.get('final_time', 10.0):.17g}
   min_residue  0.0
   reconstruct
   {{
{rec}   }}
   bc_scheme    {cfg.get('bc_scheme', 'weak')}
   liou_fix     {'yes' if cfg.get('liou_fix', False) else 'no'}
   sample_list
   {{
      groups
      {{
      }}
      free_list
      {{
{samples}
      }}
   }}
   rnd_file_loc    rnd_nos.dat
   rnd_per_sample  {int(cfg.get('rnd_per_sample', 0))}
}}

material
{{
   gamma       {cfg.get('gamma', 1.4):.17g}
   gas_const   {cfg.get('gas_const', 1.0):.17g}
   model       {model}
   viscosity
   {{
      model    constant
      mu_ref   {cfg.get('mu_ref', 0.0):.17g}
   }}
   prandtl     {cfg.get('prandtl', 0.72):.17g}
   flux        {flux}
   flux_par
   {{
      alpha      {cfg.get('ev_alpha', 0.0):.17g}
      beta       {cfg.get('ev_beta', 0.0):.17g}
   }}
   balance
   {{
       switch_active  no
       ND             yes
       HEAT           yes
       VISC           yes
   }}
}}

constants
{{
{const_text}
}}

initial_condition
{{
{ic_text}
}}

boundary
{{
{bnd_text}
}}

exact_soln
{{
   available    no
}}

integrals
{{
{force_text}
}}

output
{{
   format                vtk
   frequency             100000000
   time_stamps           {cfg.get('time_stamps', 1)}
   use_online_stat_tool  {online}
   variables
   {{
{var_text}
   }}
   surfaces
   {{
{surf_text}
   }}
   restart               {files}
   restart_frequency     100000000
   log_output            {files}
   soln_output           {files}
   save_global           {files}
   find_error            no
}}
"""


def read_dump(path: str) -> dict:
    """Parse the harness dump: records of (32-byte tag, int64 n, n doubles)."""
    out = {}
    with open(path, "rb") as fh:
        data = fh.read()
    p = 0
    while p < len(data):
        tag = data[p:p + 32].split(b"\0", 1)[0].decode()
        (n,) = struct.unpack_from("<q", data, p + 32)
        p += 40
        out[tag] = np.frombuffer(data, dtype="<f8", count=n, offset=p).copy()
        p += 8 * n
    return out


def run_case(mesh, cfg: dict, prim0: np.ndarray | None, n_steps: int, n_dump: int,
             workdir: str | None = None, timeout: float = 3600.0, rnd_rows: dict | None = None) -> dict:
    """Write the case, run the harness, return the parsed dump.

    With prim0 None the reference evaluates the parameter file's initial
    condition itself (fparser, with pert() reading rnd_rows for the first
    sample of cfg["samples"])."""
    from tensum_b200.mesh import write_part_file  # local import: tests put repo on sys.path

    if not harness_available():
        raise RuntimeError("oracle/_ref/tensum_harness is not built (make -C oracle ref)")
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="tensum_ref_")
    try:
        if own or not os.path.exists(os.path.join(wd, "PARTITION", "part_file_0.dat")):
            write_part_file(mesh, wd)
        with open(os.path.join(wd, "param.in"), "w") as fh:
            fh.write(param_text(cfg))
        if rnd_rows is not None:
            with open(os.path.join(wd, "rnd_nos.dat"), "w") as fh:
                fh.write(rnd_file_text(rnd_rows))
        ic = "-"
        if prim0 is not None:
            ic = os.path.join(wd, "ic.bin")
            np.ascontiguousarray(prim0, dtype="<f8").tofile(ic)
        out = os.path.join(wd, "dump.bin")
        env = dict(os.environ)
        env.pop("TENSUM_HARNESS_AXI", None)
        env.pop("TENSUM_HARNESS_RECON", None)
        if cfg.get("axisymmetric"):
            env["TENSUM_HARNESS_AXI"] = "1"     # the reference's -axi option
        if cfg.get("reconstruct") == "second_muscl":
            env["TENSUM_HARNESS_RECON"] = "second_muscl"
        r = subprocess.run([HARNESS, "param.in", ".", ic, str(n_steps), str(n_dump), out],
                           cwd=wd, capture_output=True, text=True, timeout=timeout, env=env)
        if r.returncode != 0 or not os.path.exists(out):
            raise RuntimeError(f"reference harness failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        if "ERROR" in r.stdout or "assertion failed" in r.stdout:
            # the reference reports configuration errors on stdout and may exit 0
            raise RuntimeError("reference harness reported an error:\n" + r.stdout[-2000:])
        return read_dump(out)
    finally:
        if own:
            import shutil
            shutil.rmtree(wd, ignore_errors=True)


def run_files(mesh, cfg: dict, prim0: np.ndarray | None, n_steps: int, timeout: float = 3600.0):
    """Run the harness in its file-output mode: the reference writes its
    solution, surface, log, force, global and restart files into SAMPLE_*/.
    Returns (dump, {file name: text}) for the files of the sample directory."""
    from tensum_b200.mesh import write_part_file

    if not harness_available():
        raise RuntimeError("oracle/_ref/tensum_harness is not built (make -C oracle ref)")
    wd = tempfile.mkdtemp(prefix="tensum_files_")
    try:
        write_part_file(mesh, wd)
        with open(os.path.join(wd, "param.in"), "w") as fh:
            fh.write(param_text(dict(cfg, files=True)))
        ic = "-"
        if prim0 is not None:
            ic = os.path.join(wd, "ic.bin")
            np.ascontiguousarray(prim0, dtype="<f8").tofile(ic)
        out = os.path.join(wd, "dump.bin")
        r = subprocess.run([HARNESS, "param.in", ".", ic, str(n_steps), "0", out, "files"],
                           cwd=wd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0 or not os.path.exists(out):
            raise RuntimeError(f"reference harness failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        if "ERROR" in r.stdout or "assertion failed" in r.stdout:
            raise RuntimeError("reference harness reported an error:\n" + r.stdout[-2000:])
        texts = {}
        for d in sorted(os.listdir(wd)):
            if d.startswith("SAMPLE_") and os.path.isdir(os.path.join(wd, d)):
                for name in sorted(os.listdir(os.path.join(wd, d))):
                    with open(os.path.join(wd, d, name)) as fh:
                        texts[name] = fh.read()
        return read_dump(out), texts
    finally:
        import shutil
        shutil.rmtree(wd, ignore_errors=True)


def rnd_file_text(rows: dict) -> str:
    """The reference's random-number file (src/fv.cc:502-551): the number of rows,
    then one row per sample: sample id followed by its random numbers."""
    lines = [str(len(rows))]
    for sid in sorted(rows):
        lines.append(" ".join([str(int(sid))] + [repr(float(x)) for x in rows[sid]]))
    return "\n".join(lines) + "\n"


def run_mc(mesh, cfg: dict, rnd_rows: dict, timeout: float = 3600.0) -> dict:
    """Run the reference's own Monte Carlo driver (FiniteVolume::run) on a case.

    cfg carries the MC keys of param_text (samples, rnd_per_sample, ic,
    online_stat=True, ...); rnd_rows maps sample id -> random numbers.  Returns
    the dump: time_instance, n_samples, m{t}_fm / m{t}_sm / m{t}_var per output
    instance (n_vertex x (5 + extras), PrimVar memory order then the extra
    variables) and prim_final (the last sample's final state).
    """
    from tensum_b200.mesh import write_part_file

    if not harness_available():
        raise RuntimeError("oracle/_ref/tensum_harness is not built (make -C oracle ref)")
    wd = tempfile.mkdtemp(prefix="tensum_mc_")
    try:
        write_part_file(mesh, wd)
        with open(os.path.join(wd, "param.in"), "w") as fh:
            fh.write(param_text(dict(cfg, online_stat=True)))
        with open(os.path.join(wd, "rnd_nos.dat"), "w") as fh:
            fh.write(rnd_file_text(rnd_rows))
        out = os.path.join(wd, "dump.bin")
        r = subprocess.run([HARNESS, "param.in", ".", "mc", "0", "0", out],
                           cwd=wd, capture_output=True, text=True, timeout=timeout)
        if r.returncode != 0 or not os.path.exists(out):
            raise RuntimeError(f"reference MC run failed ({r.returncode}):\n{r.stdout[-2000:]}\n{r.stderr[-2000:]}")
        if "ERROR" in r.stdout:
            raise RuntimeError("reference MC run reported an error:\n" + r.stdout[-2000:])
        return read_dump(out)
    finally:
        import shutil
        shutil.rmtree(wd, ignore_errors=True)
