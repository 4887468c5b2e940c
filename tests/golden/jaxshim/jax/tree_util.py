"""``jax.tree_util`` for the NumPy shim: pytrees of tuples, lists, dicts,
NamedTuples and classes registered with ``register_pytree_node_class``."""

_REGISTERED = set()


def register_pytree_node_class(cls):
    _REGISTERED.add(cls)
    return cls


def _children(node):
    if type(node) in _REGISTERED:
        children, aux = node.tree_flatten()
        return list(children), ("registered", type(node), aux)
    if isinstance(node, tuple) and hasattr(node, "_fields"):
        return list(node), ("namedtuple", type(node), None)
    if isinstance(node, (tuple, list)):
        return list(node), (type(node).__name__, type(node), None)
    if isinstance(node, dict):
        keys = sorted(node)
        return [node[k] for k in keys], ("dict", dict, keys)
    return None, None


def tree_flatten(tree):
    leaves = []

    def walk(node):
        children, spec = _children(node)
        if children is None:
            leaves.append(node)
            return ("leaf",)
        return (spec, [walk(c) for c in children])

    return leaves, walk(tree)


def tree_unflatten(spec, leaves):
    it = iter(leaves)

    def build(s):
        if s == ("leaf",):
            return next(it)
        (kind, cls, aux), kids = s
        values = [build(k) for k in kids]
        if kind == "registered":
            return cls.tree_unflatten(aux, values)
        if kind == "namedtuple":
            return cls(*values)
        if kind == "dict":
            return dict(zip(aux, values))
        return cls(values)

    return build(spec)


def tree_leaves(tree):
    return tree_flatten(tree)[0]


def tree_map(function, tree, *rest):
    leaves, spec = tree_flatten(tree)
    others = [tree_flatten(r)[0] for r in rest]
    return tree_unflatten(spec, [function(*xs) for xs in zip(leaves, *others)])
