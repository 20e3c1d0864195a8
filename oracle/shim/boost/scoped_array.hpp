#pragma once
// Intentionally empty: the compiled reference sources include it but use nothing from it.
