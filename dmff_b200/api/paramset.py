"""ParamSet: nested {field: {name: tensor}} parameters plus masks (dmff/api/paramset.py:6-163).

Tensors are torch float64 (the reference holds jax arrays); ``ParamSet`` indexes like a dict
so ``params["ADMPPmeForce"]["Q_local"]`` works on either a ParamSet or its ``.parameters``.
"""
import torch


class ParamSet:
    def __init__(self, data=None, mask=None):
        self.parameters = data if data is not None else {}
        self.mask = mask if mask is not None else {}

    def addField(self, field: str) -> None:
        if field in self.parameters:
            return
        self.parameters[field] = {}
        self.mask[field] = {}

    def addParameter(self, values, name: str, field: str = None, mask=None) -> None:
        values = torch.as_tensor(values, dtype=torch.float64)
        if mask is None:
            mask = torch.ones_like(values)
        mask = torch.as_tensor(mask, dtype=torch.float64)
        if field is not None:
            self.parameters[field][name] = values
            self.mask[field][name] = mask
        else:
            self.parameters[name] = values
            self.mask[name] = mask

    def to_torch(self):
        return self

    def __getitem__(self, key):
        return self.parameters[key]

    def __contains__(self, key):
        return key in self.parameters

    def keys(self):
        return self.parameters.keys()
