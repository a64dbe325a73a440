"""Device memory as the driver sees it (test infrastructure): the library's
stream-ordered pool (used bytes and their high-water mark) and the device's
free memory."""


class Memory:
    def __init__(self):
        from cuda.bindings import driver as d
        self.d = d
        assert d.cuInit(0)[0] == d.CUresult.CUDA_SUCCESS
        err, dev = d.cuCtxGetDevice()
        assert err == d.CUresult.CUDA_SUCCESS
        err, self.pool = d.cuDeviceGetDefaultMemPool(dev)
        assert err == d.CUresult.CUDA_SUCCESS

    def _attr(self, a):
        err, v = self.d.cuMemPoolGetAttribute(self.pool, a)
        assert err == self.d.CUresult.CUDA_SUCCESS
        return int(v)

    def reset_high(self):
        a = self.d.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH
        err, = self.d.cuMemPoolSetAttribute(self.pool, a, self.d.cuuint64_t(0))
        assert err == self.d.CUresult.CUDA_SUCCESS

    def used(self):
        return self._attr(self.d.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_CURRENT)

    def high(self):
        return self._attr(self.d.CUmemPool_attribute.CU_MEMPOOL_ATTR_USED_MEM_HIGH)

    def free(self):
        err, free, _ = self.d.cuMemGetInfo()
        assert err == self.d.CUresult.CUDA_SUCCESS
        return int(free)
