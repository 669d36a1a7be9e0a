// Empty stand-in: the regularisers compiled for the oracle need nothing from it.
#pragma once
