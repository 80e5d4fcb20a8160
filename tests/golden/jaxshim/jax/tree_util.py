"""jax.tree_util stand-in."""


def register_pytree_node(cls, flatten, unflatten):
    return None
