"""tcam dict split/recombine for autograd saving (delaunay_rasterization/internal/util.py:3-23)."""
import torch


def recombine_tensors(non_tensor_data, tensor_data):
    non_tensor_data = dict(non_tensor_data)
    tensor_keys = non_tensor_data.pop("_tensor_keys")
    out = {key: tensor for key, tensor in zip(tensor_keys, tensor_data)}
    out.update(non_tensor_data)
    return out


def split_tensors(tcam):
    tensors, keys, rest = [], [], {}
    for key, value in tcam.items():
        if isinstance(value, torch.Tensor):
            tensors.append(value)
            keys.append(key)
        else:
            rest[key] = value
    rest["_tensor_keys"] = keys
    return rest, tensors
