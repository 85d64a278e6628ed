"""``jax.lax.while_loop`` as a plain Python loop."""


def while_loop(cond_fun, body_fun, init_val):
    val = init_val
    while bool(cond_fun(val)):
        val = body_fun(val)
    return val
