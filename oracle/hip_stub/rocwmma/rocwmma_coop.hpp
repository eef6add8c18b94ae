/* stand-in for <rocwmma/rocwmma_coop.hpp>, test infrastructure only */
