"""Drop-in stage scripts for the reference pipeline (src/lagbound/pipeline.py).

The reference runs every stage as `python <_core>/<script> args` from its workspace (Workspace.run,
pipeline.py:58-76).  These scripts take the same arguments and files:

    alm_vcs.py       augmented-Lagrangian solver            (lagbound_b200/stages/alm_vcs.py)
    est_dual_vcs.py  bound estimate                         (lagbound_b200/stages/est_dual_vcs.py)
    reduce_exact.py  exact reduction                        (lagbound_b200/stages/reduce_exact.py)

install() redirects those three stages of an imported reference pipeline to the GPU scripts; every other stage
(Leiden, repair, certificate, verification) keeps running the reference's own code.  Where pymetis is not installed,
the certificate and verifier stages get lagbound_b200/dropin on their PYTHONPATH, whose pymetis module orders their
factorizations with this library's nested dissection (lb_nd_order).
"""
from __future__ import annotations

import os

HERE = os.path.dirname(os.path.abspath(__file__))
STAGES = {name: os.path.join(HERE, name) for name in ("alm_vcs.py", "est_dual_vcs.py", "reduce_exact.py")}
DROPIN = os.path.join(os.path.dirname(HERE), "dropin")
ORDERING_STAGES = ("certify_lifted_vc.py", "verify_cert.py")


def _have_pymetis():
    import importlib.util
    return importlib.util.find_spec("pymetis") is not None


def ordering_env(env=None):
    """The environment with lagbound_b200/dropin first on PYTHONPATH (its pymetis module: lb_nd_order)."""
    env = dict(env or {})
    base = env.get("PYTHONPATH", os.environ.get("PYTHONPATH", ""))
    env["PYTHONPATH"] = DROPIN + (os.pathsep + base if base else "")
    return env


def install(workspace_cls=None, vdtype=None, proximal_vdtype=None):
    """Patch Workspace.run (lagbound.pipeline.Workspace by default) so that the three stages above run the GPU
    scripts; vdtype ('f64' | 'f32' | 'bf16') sets the solver's storage of V, proximal_vdtype (default: vdtype) its
    storage in the proximal phase (the solver run that resumes the main phase's checkpoint, pipeline.py:105-136
    --resume): BF16 main phases with an FP32 proximal phase keep the certified bound within 1e-4 of FP64's.  Returns
    the original method."""
    if workspace_cls is None:
        from lagbound.pipeline import Workspace as workspace_cls
    original = workspace_cls.run

    def run(self, script, args, log, threads=None, blas_threads=None, extra_env=None):
        if script in STAGES:
            import lagbound.pipeline as P
            core = P.CORE
            try:
                P.CORE = HERE
                vd = proximal_vdtype if (proximal_vdtype and "--resume" in args) else vdtype
                args = list(args) + (["--vdtype", vd] if (vd and script == "alm_vcs.py") else [])
                return original(self, script, args, log, threads, blas_threads, extra_env)
            finally:
                P.CORE = core
        if script in ORDERING_STAGES and not _have_pymetis():
            extra_env = ordering_env(extra_env)
        return original(self, script, args, log, threads, blas_threads, extra_env)

    workspace_cls.run = run
    workspace_cls._lagbound_b200_original_run = original
    return original


def uninstall(workspace_cls=None):
    if workspace_cls is None:
        from lagbound.pipeline import Workspace as workspace_cls
    original = getattr(workspace_cls, "_lagbound_b200_original_run", None)
    if original is not None:
        workspace_cls.run = original
        del workspace_cls._lagbound_b200_original_run
