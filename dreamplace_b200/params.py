"""Global-placement parameters with the reference's defaults
(dreamplace/params.json; dreamplace/Params.py:19-34, 119-138), restricted to
the keys the global-placement hot path reads, plus ``dct_precision`` and
``recompute_field``."""
import copy
import json

DEFAULTS = {
    "gpu": 1,
    "num_bins_x": 0,
    "num_bins_y": 0,
    "global_place_stages": [{"num_bins_x": 0, "num_bins_y": 0, "iteration": 1000, "learning_rate": 0.01,
                             "wirelength": "weighted_average", "optimizer": "nesterov",
                             "Llambda_density_weight_iteration": 1, "Lsub_iteration": 1}],
    "target_density": 0.8,
    "density_weight": 8e-5,
    "random_seed": 1000,
    "gamma": 4.0,
    "ignore_net_degree": 100,
    "stop_overflow": 0.1,
    "random_center_init_flag": 1,
    "gp_noise_ratio": 0.025,
    "deterministic_flag": 0,
    "RePlAce_ref_hpwl": 350000,
    "RePlAce_LOWER_PCOF": 0.95,
    "RePlAce_UPPER_PCOF": 1.05,
    "RePlAce_skip_energy_flag": 0,
    "use_bb": 0,
    "num_threads": 8,
    "dtype": "float32",
    # Poisson-solve arithmetic of this implementation: fp32 | tf32 | bf16 | split_bf16
    "dct_precision": "split_bf16",
    # autograd path: 1 keeps only the density map between the electric
    # potential's forward and backward and recomputes the field maps there
    "recompute_field": 0,
}


class Params(object):
    """Attribute-style parameter set; unknown keys are kept as given."""

    def __init__(self, **overrides):
        for k, v in copy.deepcopy(DEFAULTS).items():
            setattr(self, k, v)
        for k, v in overrides.items():
            setattr(self, k, v)

    @classmethod
    def load(cls, path):
        with open(path) as f:
            return cls(**json.load(f))

    def todict(self):
        return dict(self.__dict__)
