"""eplace_b200 -- a B200-native engine for the ePlace / ePlace-MS global
placement inner loop (density scatter, DCT Poisson solve, field gather,
weighted-average wirelength gradient, Nesterov step with Lipschitz step
prediction), exposed through the C-ABI in include/eplace_gpu.h and mirrored
here with the reference's EPlacer_2D / EplaceNesterovOpt call surface."""
