"""``python -m canard_b200 [input.canard] [--precision fp32] [--dir D]``: runs
the reference's input file on the device path (canard_b200.driver).
``--plan-devices N`` prints its ranks placed on N devices instead."""
import argparse

from . import api, driver


def main():
    p = argparse.ArgumentParser(prog="python -m canard_b200")
    p.add_argument("input", nargs="?", default="input.canard")
    p.add_argument("--dir", default=None, help="run directory (default: the input's directory)")
    p.add_argument("--precision", default="fp64", choices=["fp64", "fp32"])
    p.add_argument("--inviscid", action="store_true", help="the reference built without VISCOUS")
    p.add_argument("--max-steps", type=int, default=None)
    p.add_argument("--split", action="store_true", help="run the input's sub-domains (nbpc) as its ranks")
    p.add_argument("--plan-devices", type=int, default=0, metavar="N",
                   help="print the input's ranks placed on N devices and the bytes they exchange; no run")
    a = p.parse_args()
    prec = api.FP32_MIXED if a.precision == "fp32" else api.FP64
    if a.plan_devices:
        driver.plan_devices(a.input, a.plan_devices, viscous=0 if a.inviscid else 1, precision=prec)
        return
    driver.run(a.input, a.dir, precision=api.FP32_MIXED if a.precision == "fp32" else api.FP64,
               viscous=0 if a.inviscid else 1, max_steps=a.max_steps, split=a.split)


if __name__ == "__main__":
    main()
