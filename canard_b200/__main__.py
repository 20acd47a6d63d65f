"""``python -m canard_b200 [input.canard] [--precision fp32] [--dir D]``: runs
the reference's input file on the device path (canard_b200.driver).
``--plan-devices N`` prints its ranks placed on N devices instead. Options not
given on the command line come from the input's ``&nml_gpu`` group."""
import argparse

from . import api, driver


def main():
    p = argparse.ArgumentParser(prog="python -m canard_b200")
    p.add_argument("input", nargs="?", default="input.canard")
    p.add_argument("--dir", default=None, help="run directory (default: the input's directory)")
    p.add_argument("--precision", default=None, choices=["fp64", "fast", "fp32"],
                   help="default: &nml_gpu nprecision, else fp64")
    p.add_argument("--inviscid", action="store_true", default=None,
                   help="the reference built without VISCOUS (default: &nml_gpu linviscid)")
    p.add_argument("--max-steps", type=int, default=None, help="default: &nml_gpu nsteps, if positive")
    p.add_argument("--split", action="store_true", default=None,
                   help="run the input's sub-domains (nbpc) as its ranks (default: &nml_gpu lsplit)")
    p.add_argument("--plan-devices", type=int, default=0, metavar="N",
                   help="print the input's ranks placed on N devices and the bytes they exchange; no run")
    a = p.parse_args()
    prec = None if a.precision is None else {"fp32": api.FP32_MIXED, "fast": api.FP64_FAST}.get(a.precision, api.FP64)
    visc = None if a.inviscid is None else 0
    if a.plan_devices:
        driver.plan_devices(a.input, a.plan_devices, viscous=visc, precision=prec)
        return
    driver.run(a.input, a.dir, precision=prec, viscous=visc, max_steps=a.max_steps, split=a.split)


if __name__ == "__main__":
    main()
