// stdp_args.h -- plastic projection kernels (pair STDP, eager substrate).
#pragma once
