"""Shared test helpers: golden fixtures, oracle inputs from a netlist."""
import os

import numpy as np

from eplace_b200.synth import Netlist

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DESIGNS = ("ref_smoke", "stdcell_2k", "mixed_5k")


def load_golden(name):
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: z[k] for k in z.files}


def golden_netlist(g):
    kw = {k[3:]: g[k] for k in g if k.startswith("nl_")}
    return Netlist(name="golden", target_density=float(g["target_density"]), bins=0, **kw)


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


class OracleDesign:
    """Object arrays in the engine's order (nodes, then fillers) for the oracle."""

    def __init__(self, nl, is_macro, num_fillers, filler_w, filler_h, core, bins, step, td):
        from oracle import oracle as O
        self.O = O
        self.nl = nl
        nf = int(num_fillers)
        self.nf = nf
        self.n = nl.num_nodes + nf
        self.w = np.concatenate([nl.node_w, np.full(nf, filler_w, np.float32)]).astype(np.float32)
        self.h = np.concatenate([nl.node_h, np.full(nf, filler_h, np.float32)]).astype(np.float32)
        self.flags = np.concatenate([np.asarray(is_macro, np.uint8) * O.MACRO,
                                     np.full(nf, O.FILLER, np.uint8)]).astype(np.uint8)
        self.grid = O.make_grid(bins[0], bins[1], core, step[0], step[1], td)
        owner = nl.pin_owner.astype(np.int64).copy()
        owner[owner >= nl.num_nodes] += nf
        self.nl_obj = nl.with_positions(nl.node_cx, nl.node_cy)
        self.nl_obj.pin_owner = owner.astype(np.int32)
        self.ppo = np.bincount(owner, minlength=self.n + nl.num_terminals)[:self.n].astype(np.int32)
        self.tcx = (nl.term_llx + np.float32(0.5) * nl.term_w).astype(np.float32)
        self.tcy = (nl.term_lly + np.float32(0.5) * nl.term_h).astype(np.float32)
        self.term, self.base = O.terminal_base_density(self.grid, nl)
        self.area = (self.w * self.h).astype(np.float32)

    @classmethod
    def from_golden(cls, g):
        nl = golden_netlist(g)
        core = (g["info_core_llx"], g["info_core_lly"], g["info_core_urx"], g["info_core_ury"])
        return cls(nl, g["node_is_macro"], g["info_num_fillers"], g["info_filler_w"], g["info_filler_h"],
                   core, (int(g["info_bins_x"]), int(g["info_bins_y"])),
                   (g["info_bin_step_x"], g["info_bin_step_y"]), float(g["target_density"]))

    def bin_area(self):
        return np.float64(np.float32(self.grid.step_x) * np.float32(self.grid.step_y))

    def evaluate(self, cx, cy, lam, exp_mode=0, qscale=0.0):
        """One totalGradientUpdate in FP64 -> dict of every intermediate."""
        O = self.O
        nd, fd, nq, fq = O.scatter(self.grid, cx, cy, self.w, self.h, self.flags, qscale)
        rho = (nd + self.base + fd + self.term) / self.bin_area()
        ex, ey, phi = O.poisson(rho, self.grid.step_x, self.grid.step_y)
        gd = O.gather(self.grid, cx, cy, self.w, self.h, ex, ey)
        tau = O.overflow(self.grid, nd, self.term, self.base, self.std_area(), self.macro_area())
        igx, igy = O.inv_gamma(tau, self.grid.step_x, self.grid.step_y)
        wl, hp, gwl = O.wirelength_grad(self.nl_obj, cx, cy, self.tcx, self.tcy, igx, igy, exp_mode)
        g = O.combine(self.ppo, self.area, self.flags, lam, gd, gwl)
        return dict(node=nd, filler=fd, node_q=nq, filler_q=fq, rho=rho, ex=ex, ey=ey, phi=phi,
                    gd=gd, gwl=gwl, tau=tau, igx=igx, igy=igy, wl=wl, hpwl=hp, g=g)

    def _area_sum(self, macro):
        # sequential float accumulation in node order, as fillerInitialization does
        m = (self.flags[:self.nl.num_nodes] & self.O.MACRO) != 0
        a = self.area[:self.nl.num_nodes][m == macro]
        return float(np.cumsum(a, dtype=np.float32)[-1]) if a.size else 0.0

    def std_area(self):
        return self._area_sum(False)

    def macro_area(self):
        return self._area_sum(True)
