"""Compile a user's get_field to LTO-IR for linking into the sm_100a kernels.

The reference's only extension point is ``get_field(time_sample, sweep_parameters, field_sample)``
(spinsim/__init__.py:381-389), jitted as a numba device function and inlined into its kernels
(I:620).  Here the same Python function is compiled by numba's CUDA target into LTO-IR behind a C-ABI
shim

    extern "C" __device__ void spinsim_user_field(double t, double* sweep_parameters, int64_t n,
                                                  double* field_sample /* 8 doubles, pre-zeroed */)

and the CUDA library links it into the time-evolution kernel with nvJitLink, so it is inlined there
just as numba inlined it into the reference's kernel.  The shim turns the raw pointers into numba
arrays with an intrinsic (no allocation), so the user function sees the same array arguments as in
the reference.  The field buffer always holds 8 doubles, so a field that writes the quadratic-shift
entry (index 3) for spin half stays in bounds.
"""
import contextlib
import threading
import weakref

_cache = weakref.WeakKeyDictionary()
_lock = threading.Lock()
CC = (10, 0)


@contextlib.contextmanager
def _device_for_typing():
    """numba types device-function calls for the current device; without a GPU (a build or test
    machine) answer with compute capability 10.0 so the LTO-IR can still be produced."""
    from numba import cuda
    import numba.cuda.dispatcher as disp
    if cuda.is_available():
        yield
        return

    class _Dev:
        compute_capability = CC

    old = disp.get_current_device
    disp.get_current_device = lambda: _Dev()
    try:
        yield
    finally:
        disp.get_current_device = old


def _ptr_as_array():
    from numba import types
    from numba.core.extending import intrinsic
    from numba.np.arrayobj import make_array, populate_array

    @intrinsic
    def ptr_as_array(typingctx, ptr, n):
        arrty = types.Array(ptr.dtype, 1, "C")
        sig = arrty(ptr, n)

        def codegen(context, builder, signature, args):
            data, count = args
            ary = make_array(arrty)(context, builder)
            itemsize = context.get_abi_sizeof(context.get_data_type(arrty.dtype))
            size = context.get_constant(types.intp, itemsize)
            populate_array(ary, data=data, shape=[count], strides=[size], itemsize=size, meminfo=None)
            return ary._getvalue()

        return sig, codegen

    return ptr_as_array


def compile_ltoir(get_field):
    """Return the LTO-IR bytes of the shim around ``get_field`` (cached per function)."""
    key = get_field
    with _lock:
        if key in _cache:
            return _cache[key]
    import numba
    from numba import cuda, types

    py_func = getattr(get_field, "py_func", get_field)
    ptr_as_array = _ptr_as_array()
    with _device_for_typing():
        user = get_field if isinstance(get_field, cuda.dispatcher.CUDADispatcher) else \
            cuda.jit(device=True, inline=True)(py_func)

        def spinsim_user_field_shim(time_sample, params, n_params, field):
            user(time_sample, ptr_as_array(params, n_params), ptr_as_array(field, 8))

        sig = types.void(types.float64, types.CPointer(types.float64), types.int64, types.CPointer(types.float64))
        ltoir, _ = cuda.compile(spinsim_user_field_shim, sig, device=True, abi="c",
                                abi_info={"abi_name": "spinsim_user_field"}, output="ltoir", cc=CC)
    _ = numba  # imported for its side effect of registering the CUDA target
    with _lock:
        _cache[key] = bytes(ltoir)
    return _cache[key]
