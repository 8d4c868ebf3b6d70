"""CPU oracle of the Warpstore hot-path operators — test infrastructure only (the parity checker and
the timed CPU baseline); the product library never imports or calls it."""
